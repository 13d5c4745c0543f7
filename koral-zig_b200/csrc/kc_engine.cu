// kc_engine.cu — libkoralcuda: the host side of the sm_100a step engine and
// its C ABI (include/koralcuda.h). One engine instance owns one CUDA stream
// and all device state of one Sim; Sim.step (koral/sim.zig:1792) becomes a
// fixed sequence of kernel launches on that stream with no host round trip
// until the step's scalars are read back at its end.
#include <math.h>

#include <cmath>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "kc_kernels.cuh"
#include "../../include/koral/kdump.h"
#include "../../include/koral/kinit.h"

using namespace kp;
using namespace kc;

namespace {

const int TPB = 128;
inline unsigned nblk(long n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

template <class Fn>
void host_par(long lo, long hi, Fn fn) {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 32) nt = 32;
  std::vector<std::thread> th;
  long n = hi - lo;
  for (unsigned w = 0; w < nt; ++w) {
    long a = lo + n * w / nt, b = lo + n * (w + 1) / nt;
    th.emplace_back([=]() {
      for (long i = a; i < b; ++i) fn(i);
    });
  }
  for (auto& x : th) x.join();
}

}  // namespace

struct kc_handle {
  kc_grid kg;
  kc_options opt;
  SimParams sp;
  DGrid gr;
  DevState ds;
  DevScalars* dsc = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  // stage buffers (koral/sim.zig:220)
  double *ut0 = nullptr, *ut1 = nullptr, *ut2 = nullptr, *dut1 = nullptr, *dut2 = nullptr, *drt1 = nullptr,
         *drt2 = nullptr, *uforget = nullptr, *staging = nullptr;
  int* flag_staging = nullptr;
  // step scalars (koral/sim.zig:237-293)
  double t = 0, dt = 0, own_dt = 0, tstepdenmax = 0, tstepdenmin = 1.0e50;
  double min_dx = 0, min_dy = 0, min_dz = 0;
  int impl_blocks = 0;  // resident blocks of the persistent implicit kernel
  double* init_dv = nullptr;  // the PUFFY init's per-column torus profile
  // block sizes of the per-cell implicit, face-flux and u2p kernels (kc_autotune)
  int tpb_implicit = TPB, tpb_flux = TPB, tpb_u2p = TPB;
#ifndef KC_IMPLICIT_PHI_FASTEST
#define KC_IMPLICIT_PHI_FASTEST 1
#endif
#ifndef KC_U2P_PHI_FASTEST
#define KC_U2P_PHI_FASTEST 0
#endif
  // thread -> cell order of the per-cell implicit and u2p kernels: on 3D grids
  // phi fastest (warps of cells sharing r and theta) or x fastest; for the
  // implicit kernel on 2D grids the same switch selects theta fastest
  int implicit_phi_fastest = KC_IMPLICIT_PHI_FASTEST, u2p_phi_fastest = KC_U2P_PHI_FASTEST;
  // the step's dt-derived coefficients: pinned host table and its device copy
  // (DevState::coef); slots 0-3 are fixed by run_step, later ones appended
  double* coef_host = nullptr;
  double* coef_dev = nullptr;
  int ncoef = 0;
  DevScalars* dsc_init = nullptr;  // the step-start value of the device scalars
  // CUDA graph of the whole step (kc_set_graph): captured once per launch
  // sequence and replayed; any setter that changes the sequence drops it
  bool use_graph = false, graph_warm = false;
  cudaGraphExec_t gexec = nullptr;
  long long graph_launches = 0;
  // the split form's list of cells left by the opening kernel
  unsigned long long* split_count = nullptr;
  int* split_cell = nullptr;
  double* split_pp0 = nullptr;
  int split_blocks = 0;  // resident blocks of the ladder kernel
  // the learned initial guess (KC_GUESS_MLP): FP32 blob, BF16 weight copies,
  // the per-cell seeded starts, and the training-pair harvest buffers
  int guess_mode = KC_GUESS_PLAIN;
  float* mlp_blob = nullptr;
  __nv_bfloat16 *mlp_w1 = nullptr, *mlp_w2 = nullptr, *mlp_w3 = nullptr;
  double* guess = nullptr;
  unsigned long long* imp_ctr = nullptr;  // [0] seeded-ladder fallbacks, [1] harvested pairs
  float *hx = nullptr, *ht = nullptr;
  long hcap = 0;
  // scalar diagnostics: fold outputs and counts, and the BL geometry of the
  // luminosity shell (built on the host at first use for that shell)
  double* diag = nullptr;
  long lum_ix = -1;
  Geom* lum_gbl = nullptr;
  double* lum_w = nullptr;
  // per-pass device time (koral/sim/timers.zig PassTimers), off by default:
  // an event is recorded at every pass boundary, and the interval up to the
  // next event belongs to the innermost pass open at the first (self time)
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_pass;
  int pass_stack[8] = {};
  int pass_depth = 0;
  double pass_ms[KC_NPASS] = {};
  long long pass_calls[KC_NPASS] = {};
  long long n_launch = 0;  // kernels launched by step passes since create
  long long nstep = 0, n_fail = 0, n_fail_step = 0, n_iters = 0, n_solves = 0, n_guard = 0;
  std::string err;
  int last_status = 0;
};

namespace {

// A rejected argument (unknown mode, bad file, short buffer): the message is
// kept for kc_last_error, but the handle stays usable.
int reject(kc_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}
// A failure of the device state (a CUDA error, a failed pass): every later
// step call returns it.
int fail(kc_handle* h, int code, const std::string& msg) {
  if (h) {
    h->err = msg;
    h->last_status = code;
  }
  return code;
}
int cuda_check(kc_handle* h, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return KC_OK;
  return fail(h, KC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
template <class T>
T* dalloc(kc_handle* h, size_t n, int& st) {
  void* p = nullptr;
  if (st) return nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T) + 16);
  if (e != cudaSuccess) {
    st = fail(h, KC_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return nullptr;
  }
  cudaMemset(p, 0, n * sizeof(T) + 16);
  h->allocs.push_back(p);
  return (T*)p;
}

// ---- metric cache, host-built once (koral/metric/precompute.zig:175) ----------
int build_cache(kc_handle* h) {
  const Grid& g = h->gr.g;
  long nc = h->gr.nc, sx = h->gr.sx, sy = h->gr.sy, sz = h->gr.sz;
  long ngh = (long)h->gr.ngx * sy * sz;
  int st = 0;
  CacheOut o;
  o.cgc = dalloc<double>(h, (size_t)NGC * nc, st);
  o.cGc = dalloc<double>(h, (size_t)NGCON * nc, st);
  o.kr = dalloc<double>(h, (size_t)NKR * nc, st);
  o.jbl = dalloc<double>(h, (size_t)16 * nc, st);
  o.blg = dalloc<double>(h, (size_t)NBL * nc, st);
  o.ngh = ngh > 0 ? ngh : 1;
  o.jb2m = dalloc<double>(h, (size_t)16 * o.ngh, st);
  for (int dim = 0; dim < 3; ++dim) {
    o.nf[dim] = h->ds.nf[dim];
    o.fgc[dim] = dalloc<double>(h, (size_t)NGC * o.nf[dim], st);
    o.fGc[dim] = dalloc<double>(h, (size_t)NGCON * o.nf[dim], st);
  }
  o.asym = dalloc<int>(h, 1, st);
  if (st) return st;
  k_cache_centers<<<nblk(nc), TPB, 0, h->stream>>>(g, h->sp.mp, sx, sy, sz, o);
  long nfc = (sx + 1) * (sy + 1) * (sz + 1);
  for (int dim = 0; dim < 3; ++dim) k_cache_faces<<<nblk(nfc), TPB, 0, h->stream>>>(g, h->sp.mp, sx, sy, sz, dim, o);
  int asym = 0;
  st = cuda_check(h, cudaMemcpyAsync(&asym, o.asym, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "metric cache");
  if (!st) st = cuda_check(h, cudaStreamSynchronize(h->stream), "metric cache");
  if (st) return st;
  if (asym) return fail(h, KC_ERR_INVALID_CONFIG, "metric cache is not bitwise symmetric where the packed layout needs it");
  h->ds.cgc = o.cgc;
  h->ds.cGc = o.cGc;
  h->ds.kr = o.kr;
  h->ds.jbl = o.jbl;
  h->ds.blg = o.blg;
  h->ds.jb2m = o.jb2m;
  for (int dim = 0; dim < 3; ++dim) {
    h->ds.fgc[dim] = o.fgc[dim];
    h->ds.fGc[dim] = o.fGc[dim];
  }
  return KC_OK;
}

// a device allocation freed at scope exit (stream-ordered work on it must have
// completed, which the init's synchronizing read-back ensures)
struct DevBufE {
  void* p = nullptr;
  ~DevBufE() {
    if (p) cudaFree(p);
  }
};

// ---- pass timers -----------------------------------------------------------------
void pass_mark(kc_handle* h) {
  size_t i = h->ev_pass.size();
  if (i == h->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    h->ev_pool.push_back(e);
  }
  cudaEventRecord(h->ev_pool[i], h->stream);
  h->ev_pass.push_back(h->pass_depth ? h->pass_stack[h->pass_depth - 1] : -1);
}
struct PassScope {
  kc_handle* h;
  bool on;
  PassScope(kc_handle* hh, int pass) : h(hh), on(hh->timing && hh->pass_depth < 8) {
    if (!on) return;
    h->pass_stack[h->pass_depth++] = pass;
    h->pass_calls[pass] += 1;
    pass_mark(h);
  }
  void end() {
    if (!on) return;
    on = false;
    --h->pass_depth;
    pass_mark(h);
  }
  ~PassScope() { end(); }
};
// after the stream has drained: fold the recorded intervals into the totals
void pass_collect(kc_handle* h) {
  for (size_t i = 0; i + 1 < h->ev_pass.size(); ++i) {
    int p = h->ev_pass[i];
    if (p < 0) continue;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, h->ev_pool[i], h->ev_pool[i + 1]) == cudaSuccess) h->pass_ms[p] += ms;
  }
  h->ev_pass.clear();
}

// ---- pass wrappers (one launch each) -----------------------------------------
int sync_check(kc_handle* h, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_check(h, e, what);
  return KC_OK;
}

BcArgs bc_args(kc_handle* h) {
  BcArgs a;
  a.bc[0] = h->sp.bc[0];
  a.bc[1] = h->sp.bc[1];
  a.bc[2] = h->sp.bc[2];
  a.gam = h->sp.gam;
  return a;
}

// C set_bc (koral/sim/bc.zig:40)
void launch_set_bc(kc_handle* h) {
  PassScope ps(h, KC_PASS_BC);
  const DGrid& gr = h->gr;
  BcArgs a = bc_args(h);
  cudaStream_t st = h->stream;
  if (gr.ngx > 0) {
    ++h->n_launch;
    k_bc_faces<<<nblk(2L * gr.ngx * gr.ny * gr.nz), TPB, 0, st>>>(h->ds, h->dsc, a, 0);
  }
  if (gr.ngy > 0) {
    ++h->n_launch;
    k_bc_faces<<<nblk(2L * gr.ngy * gr.nx * gr.nz), TPB, 0, st>>>(h->ds, h->dsc, a, 1);
  }
  if (gr.ngz > 0) {
    ++h->n_launch;
    k_bc_faces<<<nblk(2L * gr.ngz * gr.nx * gr.ny), TPB, 0, st>>>(h->ds, h->dsc, a, 2);
  }
  if (gr.ny > 1 && gr.nz == 1) {
    ++h->n_launch;
    k_corners_2d<<<1, 32, 0, st>>>(h->ds, a);
  } else if (gr.nz > 1 && gr.ny > 1) {
    long ng = gr.ng;
    const int planes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
    long nt0 = 2 * (ng - 1) + 1;
    for (const auto& pl : planes) {
      long nslice = (pl[2] == 0 ? gr.nx : pl[2] == 1 ? gr.ny : gr.nz) + 2 * ng;
      h->n_launch += 2;
      k_edge_tubes<<<nblk(4L * nslice * nt0, 64), 64, 0, st>>>(h->ds, a.gam, pl[0], pl[1], pl[2], 0);
      k_edge_tubes<<<nblk(4L * nslice, 64), 64, 0, st>>>(h->ds, a.gam, pl[0], pl[1], pl[2], 1);
    }
    ++h->n_launch;
    k_corner_cubes<<<nblk(8 * ng * ng * ng, 64), 64, 0, st>>>(h->ds, a.gam);
  }
}

void launch_calc_u2p(kc_handle* h) {
  const DGrid& gr = h->gr;
  long ndom = (long)gr.nx * gr.ny * gr.nz;
  int pnc = h->sp.correct_polaraxis ? h->sp.nccorrectpolar : 0;
  PassScope ps(h, KC_PASS_U2P);
  cudaMemsetAsync(&h->dsc->any_hd, 0, sizeof(int), h->stream);
  ++h->n_launch;
  k_u2p<<<nblk(ndom, h->tpb_u2p), h->tpb_u2p, 0, h->stream>>>(h->ds, h->dsc, h->sp.gam, h->sp.fl, h->sp.rp, pnc,
                                                                h->u2p_phi_fastest && gr.nz > 1);
  if (h->sp.do_fixups) {
    PassScope pf(h, KC_PASS_FIXUP);
    ++h->n_launch;
    k_fixup_hd<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, h->dsc, h->sp.gam, pnc);
    ++h->n_launch;
    k_fixup_apply<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, h->dsc);
  }
  launch_set_bc(h);
}

void launch_do_correct(kc_handle* h) {
  if (!h->sp.correct_polaraxis) return;
  const DGrid& gr = h->gr;
  int ncp = h->sp.nccorrectpolar;
  PassScope ps(h, KC_PASS_CORRECT);
  ++h->n_launch;
  k_polar_correct<<<nblk((long)gr.nx * gr.nz * 2 * ncp), TPB, 0, h->stream>>>(h->ds, h->sp.gam, ncp);
}

void launch_implicit(kc_handle* h, int dt_slot) {
  const DGrid& gr = h->gr;
  ImplArgs a;
  a.gam = h->sp.gam;
  a.dt_slot = dt_slot;
  a.rp = h->sp.rp;
  a.op = h->sp.op;
  a.ip = h->sp.ip;
  a.polar_nc = h->sp.correct_polaraxis ? h->sp.nccorrectpolar : 0;
  a.phi_fastest = h->implicit_phi_fastest && gr.nz > 1;
  a.y_fastest = h->implicit_phi_fastest && gr.nz == 1;
  PassScope ps(h, KC_PASS_IMPLICIT);
  // the learned guess and the harvest run in the per-cell form
  bool extra = h->guess_mode == KC_GUESS_MLP || h->hcap > 0;
  if (h->opt.implicit_mode == KC_IMPLICIT_SPLIT && !extra) {
    long ndom = (long)gr.nx * gr.ny * gr.nz;
    if (!h->split_count) {
      int st = 0;
      h->split_count = dalloc<unsigned long long>(h, 1, st);
      h->split_cell = dalloc<int>(h, ndom, st);
      h->split_pp0 = dalloc<double>(h, (size_t)NV * ndom, st);
      if (st) return;
      int dev = 0, nsm = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_implicit_ladder, TPB, 0);
      h->split_blocks = (per_sm > 0 ? per_sm : 1) * (nsm > 0 ? nsm : 1);
    }
    SplitList L = {h->split_count, h->split_cell, h->split_pp0, ndom};
    cudaMemsetAsync(h->split_count, 0, sizeof(unsigned long long), h->stream);
    ++h->n_launch;
    k_implicit_open<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, h->dsc, a, L);
    ++h->n_launch;
    k_implicit_ladder<<<h->split_blocks, TPB, 0, h->stream>>>(h->ds, h->dsc, a, L);
    return;
  }
  if (h->opt.implicit_mode == KC_IMPLICIT_COMPACTING && !extra) {
    long nwork = (long)gr.nx * (gr.ny - 2L * a.polar_nc) * gr.nz;
    if (h->impl_blocks == 0) {
      int dev = 0, nsm = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_implicit_persistent, TPB, 0);
      h->impl_blocks = (per_sm > 0 ? per_sm : 1) * (nsm > 0 ? nsm : 1);
    }
    long need = (nwork + TPB - 1) / TPB;
    int blocks = (int)(need < h->impl_blocks ? need : h->impl_blocks);
    cudaMemsetAsync(&h->dsc->work_next, 0, sizeof(unsigned long long), h->stream);
    ++h->n_launch;
    if (blocks > 0) k_implicit_persistent<<<blocks, TPB, 0, h->stream>>>(h->ds, h->dsc, a, nwork);
    return;
  }
  long ndom = (long)gr.nx * gr.ny * gr.nz;
  ImplExtra x = {nullptr, nullptr, nullptr, nullptr, 0, nullptr};
  if (h->imp_ctr) {
    x.n_fallback = h->imp_ctr;
    if (h->hcap > 0) {
      x.hx = h->hx;
      x.ht = h->ht;
      x.hcount = h->imp_ctr + 1;
      x.hcap = h->hcap;
    }
  }
  if (h->guess_mode == KC_GUESS_MLP) {
    MlpDev m = {h->mlp_w1, h->mlp_w2, h->mlp_w3, h->mlp_blob};
    ++h->n_launch;
    k_mlp_guess<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, m, a, h->guess);
    x.guess = h->guess;
  }
  ++h->n_launch;
  unsigned nb = nblk(ndom, h->tpb_implicit);
  if (extra) k_implicit<true, 2><<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, h->dsc, a, x);
  else if (a.phi_fastest) k_implicit<false, 2><<<nb, h->tpb_implicit, 0, h->stream>>>(h->ds, h->dsc, a, x);
  else k_implicit<false, 3><<<nb, h->tpb_implicit, 0, h->stream>>>(h->ds, h->dsc, a, x);
}

void launch_wavespeeds(kc_handle* h) {
  const DGrid& gr = h->gr;
  WsArgs a;
  a.gam = h->sp.gam;
  a.tsteplim = h->sp.tsteplim;
  a.op = h->sp.op;
  a.damp_nc = h->sp.dampradwavespeednearaxis;
  PassScope ps(h, KC_PASS_WAVESPEEDS);
  long n = (long)(gr.nx + 2 * (gr.nx > 1)) * (gr.ny + 2 * (gr.ny > 1)) * (gr.nz + 2 * (gr.nz > 1));
  ++h->n_launch;
  k_wavespeeds<<<nblk(n), TPB, 0, h->stream>>>(h->ds, h->dsc, a);
}

void launch_face_fluxes(kc_handle* h) {
  const DGrid& gr = h->gr;
  FluxArgs a;
  a.gam = h->sp.gam;
  a.theta = h->sp.minmod_theta;
  a.maxvel = h->sp.maxradviscvel;
  a.fl = h->sp.fl;
  a.radvisc = h->sp.radviscosity;
  long dims[3] = {gr.nx, gr.ny, gr.nz};
  PassScope ps(h, KC_PASS_FLUXES);
  for (int d = 0; d < 3; ++d) cudaMemsetAsync(h->ds.flb[d], 0, (size_t)NV * h->ds.nf[d] * 8, h->stream);
  for (int dim = 0; dim < 3; ++dim) {
    if (dims[dim] <= 1) continue;
    int c0 = dim == 0 ? 1 : 0, c1 = dim == 2 ? 1 : 2;
    long n0 = dims[c0] > 1 ? dims[c0] + 2 : dims[c0];
    long n1 = dims[c1] > 1 ? dims[c1] + 2 : dims[c1];
    long n = (dims[dim] + 1) * n0 * n1;
    ++h->n_launch;
    int tb = h->tpb_flux;
    unsigned nb = nblk(n, tb);
    bool mx = h->opt.precision == KC_MIXED;
    if (dim == 0) {
      if (mx) k_face_flux<true, 0><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
      else k_face_flux<false, 0><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
    } else if (dim == 1) {
      if (mx) k_face_flux<true, 1><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
      else k_face_flux<false, 1><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
    } else {
      if (mx) k_face_flux<true, 2><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
      else k_face_flux<false, 2><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
    }
  }
}

void launch_flux_ct(kc_handle* h) {
  const DGrid& gr = h->gr;
  long n = (long)(gr.nx + 1) * (gr.ny + 1) * (gr.nz + 1);
  PassScope ps(h, KC_PASS_FLUXCT);
  ++h->n_launch;
  if (h->opt.precision == KC_MIXED) k_ct_emf<float><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
  else k_ct_emf<double><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
  ++h->n_launch;
  if (h->opt.precision == KC_MIXED) k_ct_rebuild<float><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
  else k_ct_rebuild<double><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
}

void launch_op_explicit(kc_handle* h, int dt_slot) {
  launch_wavespeeds(h);
  launch_face_fluxes(h);
  launch_flux_ct(h);
  const DGrid& gr = h->gr;
  {
    PassScope ps(h, KC_PASS_UPDATE);
    ++h->n_launch;
    k_update<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, h->sp.gam, dt_slot);
  }
  launch_calc_u2p(h);
}

void launch_rijvisc(kc_handle* h, int dt_slot) {
  const DGrid& gr = h->gr;
  PassScope ps(h, KC_PASS_RADVISC);
  cudaMemsetAsync(h->ds.rijvisc, 0, (size_t)16 * gr.nc * 8, h->stream);
  ViscArgs a;
  a.gam = h->sp.gam;
  a.dt_slot = dt_slot;
  a.rhor = r_horizon_bl(h->sp.mp.a);
  a.alpha = h->sp.alpharadvisc;
  a.op = h->sp.op;
  long n = (long)(gr.nx + 2 * (gr.nx > 1)) * (gr.ny + 2 * (gr.ny > 1)) * (gr.nz + 2 * (gr.nz > 1));
  ++h->n_launch;
  k_rijvisc<<<nblk(n), TPB, 0, h->stream>>>(h->ds, a);
}

void launch_dynamo(kc_handle* h, int dt_slot) {
  const DGrid& gr = h->gr;
  PassScope ps(h, KC_PASS_DYNAMO);
  ++h->n_launch;
  k_scale_height<<<nblk(gr.nx, SH_WARPS), SH_WARPS * 32, 0, h->stream>>>(h->ds);
  launch_set_bc(h);
  DynArgs a;
  a.gam = h->sp.gam;
  a.dt_slot = dt_slot;
  a.a = h->sp.mp.a;
  a.rhor = r_horizon_bl(h->sp.mp.a);
  a.risco = r_isco_bl(h->sp.mp.a);
  a.dp = h->sp.dp;
  long n = (long)(gr.nx + 2 * (gr.nx > 1)) * (gr.ny + 2 * (gr.ny > 1)) * (gr.nz + 2 * (gr.nz > 1));
  ++h->n_launch;
  k_dynamo_delta_a<<<nblk(n), TPB, 0, h->stream>>>(h->ds, h->dsc, a);
  long my = gr.ny == 1 ? 1 : gr.ny + 1, mz = gr.nz == 1 ? 1 : gr.nz + 1;
  ++h->n_launch;
  k_corner_avg_a<<<nblk((long)(gr.nx + 1) * my * mz, 256), 256, 0, h->stream>>>(h->ds, h->ds.dyn_a, 1);
  ++h->n_launch;
  k_curl_apply<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, h->sp.gam, 0);
  launch_calc_u2p(h);
}

void launch_stage_deriv(kc_handle* h, double* dst, const double* a, const double* b, int delta) {
  const DGrid& gr = h->gr;
  PassScope ps(h, KC_PASS_STAGE);
  ++h->n_launch;
  k_stage_deriv<<<nblk((long)gr.nx * gr.ny * gr.nz, 256), 256, 0, h->stream>>>(h->ds, dst, a, b, delta);
}
void launch_stage_combine(kc_handle* h, double* dst, const double* a, int f1, const double* b, int f2,
                          const double* c) {
  const DGrid& gr = h->gr;
  PassScope ps(h, KC_PASS_STAGE);
  ++h->n_launch;
  k_stage_combine<<<nblk((long)gr.nx * gr.ny * gr.nz, 256), 256, 0, h->stream>>>(h->ds, dst, a, f1, b, f2, c);
}
void copy_field(kc_handle* h, double* dst, const double* src) {
  PassScope ps(h, KC_PASS_STAGE);
  cudaMemcpyAsync(dst, src, (size_t)NV * h->gr.nc * 8, cudaMemcpyDeviceToDevice, h->stream);
}

// Coefficient slots of a step (run_step fills 0-3 before its first launch)
enum { C_DT = 0, C_DT_GAM = 1, C_DT_1M2GAM = 2, C_DT_HALF = 3, NCOEF = 16 };
// the slot holding v (bit-equal), appended and copied to the device if new;
// a full table waits for the stream before it is reused (the host table is
// pinned and read by copies when they run)
int coef_slot(kc_handle* h, double v) {
  for (int i = 0; i < h->ncoef; ++i)
    if (memcmp(&h->coef_host[i], &v, 8) == 0) return i;
  if (h->ncoef == NCOEF) {
    cudaStreamSynchronize(h->stream);
    h->ncoef = 0;
  }
  int i = h->ncoef++;
  h->coef_host[i] = v;
  cudaMemcpyAsync(h->coef_dev + i, h->coef_host + i, 8, cudaMemcpyHostToDevice, h->stream);
  return i;
}
// the step's table: written on the host (no copy pending: the previous step
// ended with a stream synchronize), copied by the step's first operation
void coef_set_step(kc_handle* h, double dt) {
  h->coef_host[C_DT] = dt;
  h->coef_host[C_DT_GAM] = dt * KP_GAM_IMEX;
  h->coef_host[C_DT_1M2GAM] = dt * KP_ONE_M2GAM;
  h->coef_host[C_DT_HALF] = dt / 2.0;
  h->ncoef = 4;
}
void coef_copy_step(kc_handle* h) {
  cudaMemcpyAsync(h->coef_dev, h->coef_host, 4 * 8, cudaMemcpyHostToDevice, h->stream);
}

void reset_step_scalars(kc_handle* h) {
  cudaMemcpyAsync(h->dsc, h->dsc_init, sizeof(DevScalars), cudaMemcpyDeviceToDevice, h->stream);
}

// read the device scalars, fold them into the handle (sim.zig:634 reduceStepGlobals)
int collect_step_scalars(kc_handle* h, bool fold_cfl) {
  DevScalars z;
  cudaError_t e = cudaMemcpyAsync(&z, h->dsc, sizeof(z), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_check(h, e, "step");
  if (fold_cfl) {
    if (z.tsd_max_bits) {
      double m;
      memcpy(&m, &z.tsd_max_bits, 8);
      if (m > h->tstepdenmax) h->tstepdenmax = m;
    }
    double n;
    memcpy(&n, &z.tsd_min_bits, 8);
    if (n < h->tstepdenmin) h->tstepdenmin = n;
  }
  h->n_fail += (long long)z.n_fail;
  h->n_iters += (long long)z.n_iters;
  h->n_solves += (long long)z.n_solves;
  h->n_guard += (long long)z.n_guard;
  if (z.err) {
    char buf[128];
    snprintf(buf, sizeof buf, "device pass failed with status %d at cell %lld", z.err, z.err_cell);
    return fail(h, z.err, buf);
  }
  return KC_OK;
}

// The launch sequence of Sim.step (koral/sim.zig:1792), coefficients from the
// step table (C_* slots)
void enqueue_step(kc_handle* h) {
  coef_copy_step(h);
  reset_step_scalars(h);
  double* u = h->ds.u;
  if (h->sp.radviscosity) launch_rijvisc(h, C_DT);
  // 1st implicit
  copy_field(h, h->ut0, u);
  launch_implicit(h, C_DT_GAM);
  launch_stage_deriv(h, h->drt1, u, h->ut0, C_DT_GAM);
  // 1st explicit
  copy_field(h, h->ut1, u);
  launch_calc_u2p(h);
  launch_do_correct(h);
  launch_set_bc(h);
  launch_op_explicit(h, C_DT);
  if (h->sp.dynamo) launch_dynamo(h, C_DT);
  {
    const DGrid& gr = h->gr;
    PassScope ps(h, KC_PASS_STAGE);
    ++h->n_launch;
    k_copy_entropy_count<<<nblk((long)gr.nx * gr.ny * gr.nz, 256), 256, 0, h->stream>>>(h->ds);
  }
  launch_stage_deriv(h, h->dut1, u, h->ut1, C_DT);
  launch_stage_combine(h, u, h->ut0, C_DT, h->dut1, C_DT_1M2GAM, h->drt1);
  // 2nd implicit
  copy_field(h, h->uforget, u);
  launch_calc_u2p(h);
  launch_do_correct(h);
  launch_implicit(h, C_DT_GAM);
  launch_stage_deriv(h, h->drt2, u, h->uforget, C_DT_GAM);
  // 2nd explicit
  copy_field(h, h->ut2, u);
  launch_calc_u2p(h);
  launch_do_correct(h);
  launch_set_bc(h);
  launch_op_explicit(h, C_DT);
  if (h->sp.dynamo) launch_dynamo(h, C_DT);
  launch_stage_deriv(h, h->dut2, u, h->ut2, C_DT);
  launch_stage_combine(h, u, h->ut0, C_DT_HALF, h->dut1, C_DT_HALF, h->dut2);
  launch_stage_combine(h, u, u, C_DT_HALF, h->drt1, C_DT_HALF, h->drt2);
  launch_calc_u2p(h);
  launch_do_correct(h);
  launch_set_bc(h);
  {
    const DGrid& gr = h->gr;
    PassScope ps(h, KC_PASS_ENTROPY);
    ++h->n_launch;
    k_update_entropy<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, h->sp.gam);
  }
}

void drop_graph(kc_handle* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  h->gexec = nullptr;
  h->graph_warm = false;
}

// Enqueues one step: eagerly, or as a replay of the captured step graph. The
// graph holds the coefficient copy from the pinned table, so a replay runs
// with the values coef_set_step wrote. After any change of the launch sequence
// one step runs eagerly (lazy allocations happen outside a capture), the next
// one is captured, and later ones replay it.
int launch_step(kc_handle* h) {
  bool graph = h->use_graph && !h->timing;
  if (!graph) {
    enqueue_step(h);
    return KC_OK;
  }
  if (h->gexec) {
    h->n_launch += h->graph_launches;
    return cuda_check(h, cudaGraphLaunch(h->gexec, h->stream), "graph launch");
  }
  if (!h->graph_warm) {
    enqueue_step(h);
    h->graph_warm = true;
    return KC_OK;
  }
  int st = cuda_check(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
  if (st) return st;
  long long n0 = h->n_launch;
  enqueue_step(h);
  cudaGraph_t g = nullptr;
  st = cuda_check(h, cudaStreamEndCapture(h->stream, &g), "graph capture");
  if (!st) st = cuda_check(h, cudaGraphInstantiate(&h->gexec, g, 0), "graph instantiate");
  if (g) cudaGraphDestroy(g);
  if (st) {
    h->gexec = nullptr;
    return st;
  }
  h->graph_launches = h->n_launch - n0;
  return cuda_check(h, cudaGraphLaunch(h->gexec, h->stream), "graph launch");
}

// Sim.step (koral/sim.zig:1792)
int run_step(kc_handle* h, double forced_dt, kc_step_info* info) {
  double t = h->t;
  h->own_dt = 1.0 / h->tstepdenmax;
  double dt = isnan(forced_dt) ? h->own_dt : forced_dt;
  h->dt = dt;
  long long fail0 = h->n_fail;
  h->tstepdenmax = -1.0;
  h->tstepdenmin = 1.0e50;
  coef_set_step(h, dt);
  PassScope pstep(h, KC_PASS_STEP);
  int st = launch_step(h);
  pstep.end();
  if (st) return st;
  st = sync_check(h, "step launch");
  if (st) return st;
  st = collect_step_scalars(h, true);
  if (h->timing) pass_collect(h);
  h->t = t + dt;
  h->n_fail_step = h->n_fail - fail0;
  h->nstep += 1;
  if (info) {
    info->dt = dt;
    info->nan_cell = -1;
  }
  return st;
}

// The limotorus profile of (x1, x2) columns [c0, c0 + n) (tools.c
// init_dsandvels_limotorus, puffy.zig:572: angular-momentum root finding and
// the adaptive GK21 quadrature of ln f), one thread per column; each thread's
// quadrature segment table is its slice of `seg` (4 kMaxSeg doubles).
__global__ void __launch_bounds__(128) k_init_columns(Grid g, MetricParams mp, kcinit::TorusConsts tc,
                                                      kcinit::PuffyPhysics ph, long c0, long n, double* dvcol,
                                                      double* seg) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  long col = c0 + k, ix = col % g.nx, iy = col / g.nx;
  Geom gb0;
  geometry_bl_at(g, mp, ix, iy, 0, gb0);
  kcinit::DsVels dv = kcinit::init_dsandvels_s(gb0.xx[1], gb0.xx[2], mp.a, tc, ph, seg + k * 4L * kcinit::kMaxSeg);
  dvcol[3 * col] = dv.rho;
  dvcol[3 * col + 1] = dv.uu;
  dvcol[3 * col + 2] = dv.ell;
}

// PUFFY per-cell initial state (puffy.zig:715 prepInitCellWith, then the
// entropy and p2u of initCell, sim.zig:672) on the device, one thread per
// domain cell, from the host's per-column torus profile dv[3 (ix + nx iy)]
// (rho, u, ell of init_dsandvels). Ghost cells are left at zero.
__global__ void __launch_bounds__(128) k_init_cells(DevState s, DevScalars* sc, Grid g, MetricParams mp,
                                                    const double* dvcol,
                                                    SimParams sp, kcinit::PuffyPhysics ph, double perturb,
                                                    double perturb_rho, uint64_t seed) {
  long nx = g.nx, ny = g.ny, nd = nx * ny * g.nz;
  long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nd) return;
  long ix = d % nx, iy = (d / nx) % ny, iz = d / (nx * ny);
  double x[4] = {0.0, grid_xc(g, ix), grid_yc(g, iy), grid_zc(g, iz)};
  Geom geo, gbl;
  geometry_at(MKS2, mp, x, geo);
  geometry_bl_at(g, mp, ix, iy, iz, gbl);
  double jac[4][4];
  double xbl[4] = {0.0, gbl.xx[1], gbl.xx[2], gbl.xx[3]};
  dxdx(xbl, BL, MKS2, mp, jac);
  long col = ix + nx * iy;
  kcinit::DsVels dv = {dvcol[3 * col], dvcol[3 * col + 1], dvcol[3 * col + 2]};
  double pp[NV], uu[NV];
  int e = kcinit::prep_init_cell(geo, gbl, jac, dv, sp, ph, perturb, perturb_rho, seed, pp);
  long c = cidx(s.gr, ix, iy, iz);
  if (e) {
    set_err(sc, e, c);
    return;
  }
  pp[ENTR] = s_from_u(pp[RHO], pp[UU], sp.gam);
  p2u(pp, uu, geo, sp.gam);
  store_cell(s.p, s.gr.nc, c, pp);
  store_cell(s.u, s.gr.nc, c, uu);
}

}  // namespace

// ==== C ABI ===================================================================
extern "C" {

void kc_options_puffy(kc_options* opt) { options_puffy(opt); }
void kc_grid_puffy(int32_t nx, int32_t ny, int32_t nz, kc_grid* grid) { grid_puffy(nx, ny, nz, grid); }

const char* kc_last_error(const kc_handle* h) { return h ? h->err.c_str() : "null handle"; }

int kc_create(const kc_grid* grid, const kc_options* opt, kc_handle** out) {
  if (!grid || !opt || !out) return KC_ERR_INVALID_CONFIG;
  *out = nullptr;
  const char* why = validate_config(*grid, *opt);
  kc_handle* h = new kc_handle();
  if (why) {
    fail(h, KC_ERR_INVALID_CONFIG, why);
    *out = h;
    return KC_ERR_INVALID_CONFIG;
  }
  *out = h;
  h->kg = *grid;
  h->opt = *opt;
  params_from_options(*opt, h->sp);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(h, KC_ERR_NO_DEVICE, "no CUDA device");
  if (opt->device < 0 || opt->device >= ndev) return fail(h, KC_ERR_INVALID_CONFIG, "device ordinal out of range");
  int st = cuda_check(h, cudaSetDevice(opt->device), "cudaSetDevice");
  if (st) return st;
  st = cuda_check(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (st) return st;
  Grid g = grid_init(grid->nx, grid->ny, grid->nz, grid->ng, grid->minx, grid->maxx, grid->miny, grid->maxy, grid->minz,
                     grid->maxz);
  DGrid& gr = h->gr;
  gr.g = g;
  gr.nx = g.nx;
  gr.ny = g.ny;
  gr.nz = g.nz;
  gr.ng = g.ng;
  gr.ngx = g.ngx;
  gr.ngy = g.ngy;
  gr.ngz = g.ngz;
  gr.sx = g.nx + 2 * g.ngx;
  gr.sy = g.ny + 2 * g.ngy;
  gr.sz = g.nz + 2 * g.ngz;
  gr.nc = gr.sx * gr.sy * gr.sz;
  h->ds.gr = gr;
  for (int d = 0; d < 3; ++d) h->ds.nf[d] = (gr.sx + (d == 0)) * (gr.sy + (d == 1)) * (gr.sz + (d == 2));
  st = build_cache(h);
  if (st) return st;
  long nc = gr.nc;
  h->ds.p = dalloc<double>(h, NV * nc, st);
  h->ds.u = dalloc<double>(h, NV * nc, st);
  h->ds.flags = dalloc<int>(h, 6 * nc, st);
  h->ds.amax = dalloc<double>(h, 6 * nc, st);
  for (int d = 0; d < 3; ++d) h->ds.flb[d] = dalloc<double>(h, NV * h->ds.nf[d], st);
  for (int d = 0; d < 3; ++d) h->ds.emf[d] = dalloc<double>(h, (size_t)(gr.nx + 1) * (gr.ny + 1) * (gr.nz + 1), st);
  h->ds.rijvisc = dalloc<double>(h, 16 * nc, st);
  h->ds.dyn_a = dalloc<double>(h, nc, st);
  h->ds.vecpot = dalloc<double>(h, 6 * nc, st);
  h->ds.scaleth = dalloc<double>(h, gr.nx, st);
  h->ds.fix_p = dalloc<double>(h, NV * nc, st);
  h->ds.fix_u = dalloc<double>(h, NV * nc, st);
  h->ut0 = dalloc<double>(h, NV * nc, st);
  h->ut1 = dalloc<double>(h, NV * nc, st);
  h->ut2 = dalloc<double>(h, NV * nc, st);
  h->dut1 = dalloc<double>(h, NV * nc, st);
  h->dut2 = dalloc<double>(h, NV * nc, st);
  h->drt1 = dalloc<double>(h, NV * nc, st);
  h->drt2 = dalloc<double>(h, NV * nc, st);
  h->uforget = dalloc<double>(h, NV * nc, st);
  h->staging = dalloc<double>(h, NV * nc, st);
  h->flag_staging = dalloc<int>(h, 6 * nc, st);
  h->dsc = dalloc<DevScalars>(h, 1, st);
  h->dsc_init = dalloc<DevScalars>(h, 1, st);
  h->diag = dalloc<double>(h, 16, st);
  h->coef_dev = dalloc<double>(h, NCOEF, st);
  if (st) return st;
  if (cudaMallocHost(&h->coef_host, NCOEF * 8) != cudaSuccess) return fail(h, KC_ERR_OOM, "cudaMallocHost");
  memset(h->coef_host, 0, NCOEF * 8);
  h->ds.coef = h->coef_dev;
  {
    DevScalars z;
    memset(&z, 0, sizeof(z));
    double big = 1.0e50;
    memcpy(&z.tsd_min_bits, &big, 8);
    if ((st = cuda_check(h, cudaMemcpy(h->dsc_init, &z, sizeof(z), cudaMemcpyHostToDevice), "create"))) return st;
  }
  // set_grid min-size scan with C's mdx quirk (koral/sim.zig:443)
  double mdx = -1, mdy = -1, mdz = -1;
  for (long ix = 0; ix < g.nx; ++ix)
    for (long iy = 0; iy < g.ny; ++iy)
      for (long iz = 0; iz < g.nz; ++iz) {
        double dx = cell_size(g, ix, 0), dy = cell_size(g, iy, 1), dz = cell_size(g, iz, 2);
        if (dx < mdx || mdx < 0) mdx = dx;
        if (dy < mdx || mdy < 0) mdy = dy;
        if (dz < mdx || mdz < 0) mdz = dz;
      }
  h->min_dx = mdx;
  h->min_dy = mdy;
  h->min_dz = mdz;
  return cuda_check(h, cudaDeviceSynchronize(), "kc_create");
}

void kc_destroy(kc_handle* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  if (h->coef_host) cudaFreeHost(h->coef_host);
  for (void* p : h->allocs) cudaFree(p);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

static int upload_field(kc_handle* h, double* dst, const double* host, int nv) {
  if (!h || !host) return KC_ERR_INVALID_CONFIG;
  long n = (long)nv * h->gr.nc;
  int st = cuda_check(h, cudaMemcpyAsync(h->staging, host, n * 8, cudaMemcpyHostToDevice, h->stream), "upload");
  if (st) return st;
  k_aos_to_soa<<<nblk(n, 256), 256, 0, h->stream>>>(h->staging, dst, h->gr.nc, nv);
  return cuda_check(h, cudaStreamSynchronize(h->stream), "upload");
}
static int download_field(kc_handle* h, const double* src, double* host, int nv) {
  if (!h || !host) return KC_ERR_INVALID_CONFIG;
  long n = (long)nv * h->gr.nc;
  k_soa_to_aos<<<nblk(n, 256), 256, 0, h->stream>>>(src, h->staging, h->gr.nc, nv);
  int st = cuda_check(h, cudaMemcpyAsync(host, h->staging, n * 8, cudaMemcpyDeviceToHost, h->stream), "download");
  if (st) return st;
  return cuda_check(h, cudaStreamSynchronize(h->stream), "download");
}

int kc_upload_prims(kc_handle* h, const double* p) { return upload_field(h, h->ds.p, p, NV); }
int kc_upload_cons(kc_handle* h, const double* u) { return upload_field(h, h->ds.u, u, NV); }
int kc_download_prims(kc_handle* h, double* p) { return download_field(h, h->ds.p, p, NV); }
int kc_download_cons(kc_handle* h, double* u) { return download_field(h, h->ds.u, u, NV); }
int kc_upload_flags(kc_handle* h, const int32_t* f) {
  if (!h || !f) return KC_ERR_INVALID_CONFIG;
  long n = 6L * h->gr.nc;
  int st = cuda_check(h, cudaMemcpyAsync(h->flag_staging, f, n * 4, cudaMemcpyHostToDevice, h->stream), "upload");
  if (st) return st;
  k_flags_to_soa<<<nblk(n, 256), 256, 0, h->stream>>>(h->flag_staging, h->ds.flags, h->gr.nc);
  return cuda_check(h, cudaStreamSynchronize(h->stream), "upload");
}
int kc_download_flags(kc_handle* h, int32_t* f) {
  if (!h || !f) return KC_ERR_INVALID_CONFIG;
  long n = 6L * h->gr.nc;
  k_flags_to_aos<<<nblk(n, 256), 256, 0, h->stream>>>(h->ds.flags, h->flag_staging, h->gr.nc);
  int st = cuda_check(h, cudaMemcpyAsync(f, h->flag_staging, n * 4, cudaMemcpyDeviceToHost, h->stream), "download");
  if (st) return st;
  return cuda_check(h, cudaStreamSynchronize(h->stream), "download");
}

int kc_set_counters(kc_handle* h, const kc_counters* c) {
  if (!h || !c) return KC_ERR_INVALID_CONFIG;
  h->t = c->t;
  h->dt = c->dt;
  h->own_dt = c->own_dt;
  h->tstepdenmax = c->tstepdenmax;
  h->tstepdenmin = c->tstepdenmin;
  h->nstep = c->nstep;
  h->n_fail = c->n_radimp_failures;
  h->n_fail_step = c->n_radimp_fail_step;
  h->n_iters = c->n_radimp_iters;
  h->n_solves = c->n_radimp_solves;
  h->n_guard = c->n_guard_recoveries;
  return KC_OK;
}
int kc_get_counters(kc_handle* h, kc_counters* c) {
  if (!h || !c) return KC_ERR_INVALID_CONFIG;
  c->t = h->t;
  c->dt = h->dt;
  c->own_dt = h->own_dt;
  c->tstepdenmax = h->tstepdenmax;
  c->tstepdenmin = h->tstepdenmin;
  c->nstep = h->nstep;
  c->n_radimp_failures = h->n_fail;
  c->n_radimp_fail_step = h->n_fail_step;
  c->n_radimp_iters = h->n_iters;
  c->n_radimp_solves = h->n_solves;
  c->n_guard_recoveries = h->n_guard;
  return KC_OK;
}

int kc_init_timestep_guess(kc_handle* h) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  const double ws = 10000.0;
  double tsd;
  if (h->gr.nz > 1) tsd = ws / h->min_dx + ws / h->min_dy + ws / h->min_dz;
  else if (h->gr.ny > 1) tsd = ws / h->min_dx + ws / h->min_dy;
  else tsd = ws / h->min_dx;
  tsd /= h->sp.tsteplim;
  h->tstepdenmax = tsd;
  h->tstepdenmin = tsd;
  return KC_OK;
}

int kc_set_bc(kc_handle* h) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  reset_step_scalars(h);
  launch_set_bc(h);
  int st = sync_check(h, "set_bc");
  return st ? st : collect_step_scalars(h, false);
}
int kc_calc_u2p(kc_handle* h) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  reset_step_scalars(h);
  launch_calc_u2p(h);
  int st = sync_check(h, "calc_u2p");
  return st ? st : collect_step_scalars(h, false);
}
// dump.scalarRow (koral/io/dump.zig:383) with scalars.zig:225 globalScalars
namespace {
double radius_bl_at(const kc_handle* h, long ix) {
  const Grid& g = h->gr.g;
  double xx[4] = {0.0, grid_xc(g, ix), grid_yc(g, 0), grid_zc(g, 0)}, o[4];
  mks2_to_bl(xx, h->sp.mp, o);
  return o[1];
}
long shell_index(const kc_handle* h, double radius) {
  for (long ix = 0; ix < h->gr.nx; ++ix)
    if (radius_bl_at(h, ix) > radius) return ix;
  return h->gr.nx - 1;
}
}  // namespace

int kc_scalars(kc_handle* h, double dt, double r_lum, double r_scale, kc_scalar_row* out) {
  if (!h || !out) return KC_ERR_INVALID_CONFIG;
  const DGrid& gr = h->gr;
  const Grid& g = gr.g;
  const double pi = KP_PI;
  const bool twod = gr.nz == 1;
  long ix_h = shell_index(h, r_horizon_bl(h->sp.mp.a));
  long ix_l = shell_index(h, r_lum);
  long ix_s = shell_index(h, r_scale);
  long nyz = (long)gr.ny * gr.nz, ndom = (long)gr.nx * nyz;
  int st = KC_OK;
  if (h->lum_ix != ix_l) {
    // BL geometry and BL cell widths of the luminosity shell (scalars.zig:190,199)
    std::vector<Geom> gb(nyz);
    std::vector<double> w(2 * nyz);
    host_par(0, nyz, [&](long t) {
      long iy = t % gr.ny, iz = t / gr.ny;
      geometry_bl_at(g, h->sp.mp, ix_l, iy, iz, gb[t]);
      double a[4] = {0.0, grid_xc(g, ix_l), grid_yl(g, iy), grid_zc(g, iz)}, oa[4];
      double b[4] = {0.0, grid_xc(g, ix_l), grid_yl(g, iy + 1), grid_zc(g, iz)}, ob[4];
      mks2_to_bl(a, h->sp.mp, oa);
      mks2_to_bl(b, h->sp.mp, ob);
      w[t] = kmath::fabs(ob[2] - oa[2]);
      double c[4] = {0.0, grid_xc(g, ix_l), grid_yc(g, iy), grid_zl(g, iz)}, oc[4];
      double d[4] = {0.0, grid_xc(g, ix_l), grid_yc(g, iy), grid_zl(g, iz + 1)}, od[4];
      mks2_to_bl(c, h->sp.mp, oc);
      mks2_to_bl(d, h->sp.mp, od);
      w[nyz + t] = twod ? 2.0 * pi : kmath::fabs(od[3] - oc[3]) * (2.0 * pi / (g.maxz - g.minz));
    });
    if (!h->lum_gbl) h->lum_gbl = dalloc<Geom>(h, nyz, st);
    if (!h->lum_w) h->lum_w = dalloc<double>(h, 2 * nyz, st);
    if (st) return st;
    cudaMemcpy(h->lum_gbl, gb.data(), nyz * sizeof(Geom), cudaMemcpyHostToDevice);
    cudaMemcpy(h->lum_w, w.data(), 2 * nyz * sizeof(double), cudaMemcpyHostToDevice);
    h->lum_ix = ix_l;
  }
  // term buffers in the AoS staging area (unused between uploads/downloads)
  double* mass_t = h->staging;
  double* mdot_t = mass_t + ndom;
  double* rad_t = mdot_t + nyz;
  double* tot_t = rad_t + nyz;
  double* scaleth = tot_t + nyz;
  double* res = h->diag;  // mass, mdot, radlum, totallum; [8..9] counts
  reset_step_scalars(h);
  cudaMemsetAsync(res, 0, 16 * sizeof(double), h->stream);
  double phifac = gr.nz > 1 ? 2.0 * pi / (g.maxz - g.minz) : 1.0;
  k_diag_cells<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, phifac, mass_t, (unsigned long long*)(res + 8));
  double dzfac = twod ? 0.0 : 2.0 * pi / (g.maxz - g.minz);
  k_diag_mdot<<<nblk(nyz), TPB, 0, h->stream>>>(h->ds, h->dsc, ix_h, dzfac, mdot_t);
  k_diag_lum<<<nblk(nyz), TPB, 0, h->stream>>>(h->ds, h->dsc, ix_l, h->sp.gam, h->lum_gbl, h->lum_w,
                                                 h->lum_w + nyz, rad_t, tot_t);
  k_fold_ordered<<<1, 256, 0, h->stream>>>(mass_t, ndom, res + 0);
  k_fold_ordered<<<1, 256, 0, h->stream>>>(mdot_t, nyz, res + 1);
  k_fold_ordered<<<1, 256, 0, h->stream>>>(rad_t, nyz, res + 2);
  k_fold_ordered<<<1, 256, 0, h->stream>>>(tot_t, nyz, res + 3);
  // scale height: the dynamo's per-radius fold (dynamo.zig:239), into a scratch row
  DevState ds2 = h->ds;
  ds2.scaleth = scaleth;
  k_scale_height<<<nblk(gr.nx, SH_WARPS), SH_WARPS * 32, 0, h->stream>>>(ds2);
  k_init_beta_max<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, h->dsc, h->sp.gam);
  double hres[10], hsh = 0.0;
  DevScalars z;
  if ((st = sync_check(h, "scalars"))) return st;
  cudaMemcpyAsync(hres, res, sizeof hres, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&hsh, scaleth + ix_s, sizeof hsh, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(&z, h->dsc, sizeof z, cudaMemcpyDeviceToHost, h->stream);
  if ((st = cuda_check(h, cudaStreamSynchronize(h->stream), "scalars"))) return st;
  if (z.err) {
    char buf[128];
    snprintf(buf, sizeof buf, "scalars: velocity conversion failed with status %d at cell %lld", z.err, z.err_cell);
    return fail(h, z.err, buf);
  }
  unsigned long long counts[2];
  memcpy(counts, hres + 8, sizeof counts);
  double maxb = 0.0;
  if (z.tsd_max_bits) memcpy(&maxb, &z.tsd_max_bits, 8);
  out->t = h->t;
  out->dt = dt;
  out->nstep = h->nstep;
  out->mass = hres[0];
  out->mdot = -hres[1];
  out->radlum = hres[2];
  out->totallum = hres[3];
  out->scaleheight = hsh;
  out->max_pmag_ptot = maxb;
  out->n_hd_fixup = (int64_t)counts[1];
  out->n_radimp_fail = h->n_fail;
  out->n_nan = (int64_t)counts[0];
  out->n_floorguard = h->n_guard;
  return KC_OK;
}

int kc_finish_init(kc_handle* h) {
  int st = kc_set_bc(h);
  if (st) return st;
  return kc_init_timestep_guess(h);
}
int kc_cfl_dt(kc_handle* h, double* dt) {
  if (!h || !dt) return KC_ERR_INVALID_CONFIG;
  *dt = 1.0 / h->tstepdenmax;
  return KC_OK;
}
int kc_step(kc_handle* h, double forced_dt, kc_step_info* info) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (h->last_status) return h->last_status;
  return run_step(h, forced_dt, info);
}
int kc_step_n(kc_handle* h, int32_t nsteps, double forced_dt) {
  for (int i = 0; i < nsteps; ++i) {
    int st = kc_step(h, forced_dt, nullptr);
    if (st) return st;
  }
  return KC_OK;
}

// debugging surface for the parity tests: run one pass
int kc_set_pass_timing(kc_handle* h, int32_t on) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (h->pass_depth) return reject(h, KC_ERR_INVALID_CONFIG, "pass timing changed inside a pass");
  h->timing = on != 0;
  h->ev_pass.clear();
  for (int i = 0; i < KC_NPASS; ++i) {
    h->pass_ms[i] = 0.0;
    h->pass_calls[i] = 0;
  }
  return KC_OK;
}
int kc_get_pass_times(kc_handle* h, double* ms, int64_t* calls) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  for (int i = 0; i < KC_NPASS; ++i) {
    if (ms) ms[i] = h->pass_ms[i];
    if (calls) calls[i] = h->pass_calls[i];
  }
  return KC_OK;
}
const char* kc_pass_name(int32_t pass) {
  static const char* names[KC_NPASS] = {"step",  "radvisc",    "implicit", "u2p",    "fixup",  "bc",    "correct",
                                        "wavespeeds", "fluxes", "fluxct",   "update", "dynamo", "stage", "entropy"};
  return (pass >= 0 && pass < KC_NPASS) ? names[pass] : "";
}
int kc_get_stream(kc_handle* h, void** stream) {
  if (!h || !stream) return KC_ERR_INVALID_CONFIG;
  *stream = (void*)h->stream;
  return KC_OK;
}
int kc_get_launch_count(kc_handle* h, int64_t* n) {
  if (!h || !n) return KC_ERR_INVALID_CONFIG;
  *n = h->n_launch;
  return KC_OK;
}

int kc_debug_phase(kc_handle* h, int phase, double dt) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  reset_step_scalars(h);
  switch (phase) {
    case 0: launch_wavespeeds(h); break;
    case 1: launch_face_fluxes(h); break;
    case 2: launch_flux_ct(h); break;
    case 3: {
      const DGrid& gr = h->gr;
      ++h->n_launch;
      k_update<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, h->sp.gam, coef_slot(h, dt));
      break;
    }
    case 4: launch_calc_u2p(h); break;
    case 5: launch_implicit(h, coef_slot(h, dt)); break;
    case 6: launch_rijvisc(h, coef_slot(h, dt)); break;
    case 7: launch_dynamo(h, coef_slot(h, dt)); break;
    case 8: launch_do_correct(h); break;
    case 9: launch_op_explicit(h, coef_slot(h, dt)); break;
    default: return KC_ERR_INVALID_CONFIG;
  }
  int st = sync_check(h, "phase");
  if (st) return st;
  return collect_step_scalars(h, phase == 0 || phase == 9);
}
int kc_debug_get_array(kc_handle* h, int which, double* out) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  const double* src = nullptr;
  size_t n = 0;
  switch (which) {
    case 1: src = h->ds.rijvisc; n = 16 * h->gr.nc; break;
    case 2: src = h->ds.flb[0]; n = NV * h->ds.nf[0]; break;
    case 3: src = h->ds.flb[1]; n = NV * h->ds.nf[1]; break;
    case 4: src = h->ds.flb[2]; n = NV * h->ds.nf[2]; break;
    case 5: src = h->ds.scaleth; n = h->gr.nx; break;
    case 10: src = h->ds.amax; n = 6 * h->gr.nc; break;
    default: return KC_ERR_INVALID_CONFIG;
  }
  cudaMemcpy(out, src, n * 8, cudaMemcpyDeviceToHost);
  return (int)n;
}

int kc_set_precision(kc_handle* h, int32_t mode) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (mode != KC_PLAIN_FP64 && mode != KC_MIXED) return reject(h, KC_ERR_INVALID_CONFIG, "unknown precision mode");
  h->opt.precision = mode;
  drop_graph(h);
  return KC_OK;
}
int kc_set_implicit_mode(kc_handle* h, int32_t mode) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (mode != KC_IMPLICIT_PER_CELL && mode != KC_IMPLICIT_COMPACTING && mode != KC_IMPLICIT_SPLIT)
    return reject(h, KC_ERR_INVALID_CONFIG, "unknown implicit mode");
  h->opt.implicit_mode = mode;
  drop_graph(h);
  return KC_OK;
}
static int ensure_imp_ctr(kc_handle* h) {
  int st = 0;
  if (!h->imp_ctr) h->imp_ctr = dalloc<unsigned long long>(h, 2, st);
  return st;
}
// The CUDA graph form of the step (no reference counterpart): on, the whole
// step's launch sequence is captured once and replayed (bit-identical).
int kc_set_graph(kc_handle* h, int32_t on) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  h->use_graph = on != 0;
  return KC_OK;
}
int kc_set_guess(kc_handle* h, int32_t mode, const float* weights, int64_t nweights) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (mode == KC_GUESS_PLAIN) {
    h->guess_mode = KC_GUESS_PLAIN;
    drop_graph(h);
    return KC_OK;
  }
  if (mode != KC_GUESS_MLP) return reject(h, KC_ERR_INVALID_CONFIG, "unknown guess mode");
  if (!weights || nweights != KC_MLP_NWEIGHTS)
    return reject(h, KC_ERR_INVALID_CONFIG, "learned guess needs KC_MLP_NWEIGHTS floats");
  for (int64_t i = 0; i < nweights; ++i)
    if (!std::isfinite(weights[i])) return reject(h, KC_ERR_INVALID_CONFIG, "non-finite guess weight");
  for (int k = 0; k < MLP_IN; ++k)
    if (!(weights[MLP_OFF_ISTD + k] > 0.0f)) return reject(h, KC_ERR_INVALID_CONFIG, "guess input std must be > 0");
  int st = ensure_imp_ctr(h);
  const DGrid& gr = h->gr;
  long ndom = (long)gr.nx * gr.ny * gr.nz;
  if (!h->mlp_blob) {
    h->mlp_blob = dalloc<float>(h, MLP_NW, st);
    h->mlp_w1 = dalloc<__nv_bfloat16>(h, MLP_H * MLP_IN, st);
    h->mlp_w2 = dalloc<__nv_bfloat16>(h, MLP_H * MLP_H, st);
    h->mlp_w3 = dalloc<__nv_bfloat16>(h, 8 * MLP_H, st);
    h->guess = dalloc<double>(h, (size_t)NV * ndom, st);
  }
  if (st) return st;
  int e = cuda_check(h, cudaMemcpyAsync(h->mlp_blob, weights, MLP_NW * 4, cudaMemcpyHostToDevice, h->stream),
                     "guess weights");
  if (e) return e;
  k_mlp_pack<<<(MLP_H * MLP_H + 127) / 128, 128, 0, h->stream>>>(h->mlp_blob, h->mlp_w1, h->mlp_w2, h->mlp_w3);
  e = cuda_check(h, cudaStreamSynchronize(h->stream), "guess pack");
  if (e) return e;
  h->guess_mode = KC_GUESS_MLP;
  drop_graph(h);
  return KC_OK;
}
int kc_harvest_implicit(kc_handle* h, int64_t capacity) {
  if (!h || capacity < 0) return KC_ERR_INVALID_CONFIG;
  int st = ensure_imp_ctr(h);
  if (st) return st;
  if (capacity > h->hcap) {
    h->hx = dalloc<float>(h, (size_t)capacity * MLP_IN, st);
    h->ht = dalloc<float>(h, (size_t)capacity * MLP_OUT, st);
    if (st) return st;
  }
  h->hcap = capacity;
  drop_graph(h);
  return cuda_check(h, cudaMemsetAsync(h->imp_ctr + 1, 0, 8, h->stream), "harvest reset");
}
int kc_get_harvest(kc_handle* h, float* features, float* targets, int64_t capacity, int64_t* n_out) {
  if (!h || !n_out || capacity < 0) return KC_ERR_INVALID_CONFIG;
  *n_out = 0;
  if (!h->imp_ctr || h->hcap == 0) return KC_OK;
  unsigned long long cnt = 0;
  int e = cuda_check(h, cudaMemcpyAsync(&cnt, h->imp_ctr + 1, 8, cudaMemcpyDeviceToHost, h->stream), "harvest count");
  if (!e) e = cuda_check(h, cudaStreamSynchronize(h->stream), "harvest count");
  if (e) return e;
  long n = (long)cnt < h->hcap ? (long)cnt : h->hcap;
  if (n > capacity) n = capacity;
  if (n > 0 && features)
    e = cuda_check(h, cudaMemcpy(features, h->hx, (size_t)n * MLP_IN * 4, cudaMemcpyDeviceToHost), "harvest x");
  if (!e && n > 0 && targets)
    e = cuda_check(h, cudaMemcpy(targets, h->ht, (size_t)n * MLP_OUT * 4, cudaMemcpyDeviceToHost), "harvest t");
  if (e) return e;
  *n_out = n;
  return KC_OK;
}
int64_t kc_guess_fallbacks(kc_handle* h) {
  if (!h || !h->imp_ctr) return 0;
  unsigned long long v = 0;
  cudaMemcpy(&v, h->imp_ctr, 8, cudaMemcpyDeviceToHost);
  return (int64_t)v;
}
// The PUFFY init sequence (puffy.zig:873 initAllWith, then initTimestepGuess as
// problems/puffy/main.zig:304 does). The limotorus profile and the per-cell
// primitives are built on the host (one torus solve per (x1, x2) column, the
// cells of a column in parallel threads); set_bc, B from A, the second set_bc
// and the beta normalization run on the device.
int kc_init_puffy(kc_handle* h, double perturb, double perturb_rho, uint64_t seed, double* fac_out) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  const DGrid& gr = h->gr;
  const Grid& g = gr.g;
  const long nc = gr.nc;
  const MetricParams mp = h->sp.mp;
  kcinit::PuffyPhysics ph;
  ph.mass = h->opt.mass;
  kcinit::TorusConsts tc = kcinit::torus_consts(mp.a, ph);
  h->last_status = 0;
  h->err.clear();
  // the torus profile per (x1, x2) column (the metric is axisymmetric, so one
  // solve serves a column), in chunks whose quadrature scratch stays <= 1 GiB
  long ncol = (long)g.nx * g.ny;
  int st = 0;
  if (!h->init_dv) h->init_dv = dalloc<double>(h, (size_t)3 * ncol, st);
  if (st) return st;
  double* ddv = h->init_dv;
  const long chunk = 65536;
  long nseg = ncol < chunk ? ncol : chunk;
  DevBufE seg;
  if (cudaMalloc(&seg.p, (size_t)nseg * 4 * kcinit::kMaxSeg * 8) != cudaSuccess)
    return fail(h, KC_ERR_OOM, "init quadrature scratch");
  for (long c0 = 0; c0 < ncol; c0 += chunk) {
    long n = ncol - c0 < chunk ? ncol - c0 : chunk;
    k_init_columns<<<nblk(n), TPB, 0, h->stream>>>(g, mp, tc, ph, c0, n, ddv, (double*)seg.p);
  }
  st = cuda_check(h, cudaMemsetAsync(h->ds.flags, 0, 6L * nc * sizeof(int), h->stream), "init");
  if (!st) st = cuda_check(h, cudaMemsetAsync(h->ds.vecpot, 0, 6L * nc * sizeof(double), h->stream), "init");
  if (!st) st = cuda_check(h, cudaMemsetAsync(h->ds.p, 0, (size_t)NV * nc * 8, h->stream), "init");
  if (!st) st = cuda_check(h, cudaMemsetAsync(h->ds.u, 0, (size_t)NV * nc * 8, h->stream), "init");
  if (st) return st;
  const double gam = h->sp.gam;
  reset_step_scalars(h);
  k_init_cells<<<nblk((long)g.nx * g.ny * g.nz), TPB, 0, h->stream>>>(h->ds, h->dsc, g, mp, ddv, h->sp, ph, perturb,
                                                                       perturb_rho, seed);
  // a failed torus cell is reported through the device scalars' error slot
  if ((st = sync_check(h, "init")) || (st = collect_step_scalars(h, false))) return st;
  reset_step_scalars(h);
  launch_set_bc(h);
  long my = gr.ny == 1 ? 1 : gr.ny + 1, mz = gr.nz == 1 ? 1 : gr.nz + 1;
  k_corner_avg_a<<<nblk((long)(gr.nx + 1) * my * mz, 256), 256, 0, h->stream>>>(h->ds, h->ds.p + (long)B1 * nc, 0);
  k_curl_apply<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, gam, 1);
  k_init_ghost_b<<<nblk(nc), TPB, 0, h->stream>>>(h->ds, gam);
  launch_set_bc(h);
  if ((st = sync_check(h, "init")) || (st = collect_step_scalars(h, false))) return st;
  // postinit: global beta maximum, then B *= sqrt(maxbeta / maxb) over the domain
  reset_step_scalars(h);
  k_init_beta_max<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, h->dsc, gam);
  DevScalars z;
  st = cuda_check(h, cudaMemcpyAsync(&z, h->dsc, sizeof(z), cudaMemcpyDeviceToHost, h->stream), "init");
  if (!st) st = cuda_check(h, cudaStreamSynchronize(h->stream), "init");
  if (st) return st;
  double maxb = 0.0;
  if (z.tsd_max_bits) memcpy(&maxb, &z.tsd_max_bits, 8);
  double fac = kmath::sqrt(ph.maxbeta / maxb);
  k_init_beta_scale<<<nblk((long)gr.nx * gr.ny * gr.nz), TPB, 0, h->stream>>>(h->ds, gam, fac);
  if ((st = sync_check(h, "init"))) return st;
  if ((st = cuda_check(h, cudaStreamSynchronize(h->stream), "init"))) return st;
  h->t = 0.0;
  h->dt = 0.0;
  h->own_dt = 0.0;
  h->nstep = 0;
  h->n_fail = h->n_fail_step = h->n_iters = h->n_solves = h->n_guard = 0;
  if (fac_out) *fac_out = fac;
  return kc_init_timestep_guess(h);
}

}  // extern "C"

// ==== batched per-cell entry points ============================================
namespace {

// golden-record geometry: gg and GG upper triangles, gdet, alpha, gttpert
// (koral/testing/golden.zig:241 geomFromRecord)
__device__ void geom_from_record23(const double* v, Geom& g) {
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
  g.gdet = v[20];
  g.alpha = v[21];
  g.gttpert = v[22];
  for (int i = 0; i < 4; ++i) g.xx[i] = 0.0;
}

struct BatchArgs {
  double gam;
  RadParams rp;
  OpacParams op;
  ImplicitParams ip;
  FloorParams fl;
};

__global__ void __launch_bounds__(128) k_implicit_batch(long n, const double* __restrict__ geom23,
                                                        const double* __restrict__ dt, double* pp_io, int* res,
                                                        BatchArgs a, const int* order = nullptr) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  long i = order ? order[t] : t;  // the sorted form visits cells in key order
  Geom g;
  geom_from_record23(geom23 + i * 23, g);
  double pp[NV], uu[NV];
  for (int k = 0; k < NV; ++k) pp[k] = pp_io[i * NV + k];
  ImplicitResult r = solve_implicit_lab(uu, pp, g, dt[i], a.gam, a.rp, a.op, a.ip);
  for (int k = 0; k < NV; ++k) pp_io[i * NV + k] = pp[k];
  int* o = res + i * 6;
  o[0] = r.ok;
  o[1] = r.rung;
  o[2] = r.iters;
  o[3] = r.whichprim;
  o[4] = r.whicheq;
  o[5] = r.whichframe;
}

__global__ void __launch_bounds__(128) k_u2p_batch(long n, const double* __restrict__ geom23,
                                                   const double* __restrict__ uu_in, double* pp_io, int* fl_out,
                                                   BatchArgs a) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  geom_from_record23(geom23 + i * 23, g);
  double pp[NV], uu[NV];
  for (int k = 0; k < NV; ++k) {
    pp[k] = pp_io[i * NV + k];
    uu[k] = uu_in[i * NV + k];
  }
  U2pMhdRes res = u2p_mhd(uu, pp, g, a.gam, a.fl);
  U2pRadRes rr = u2p_rad(uu, pp, g, a.rp);
  int gc = 0;
  check_floors_mhd(pp, g, a.gam, a.fl, gc);
  check_floors_rad(pp, g, a.rp);
  for (int k = 0; k < NV; ++k) pp_io[i * NV + k] = pp[k];
  fl_out[i * 3 + 0] = res.entropy_used;
  fl_out[i * 3 + 1] = res.fixup;
  fl_out[i * 3 + 2] = rr.corrected ? -1 : 0;
}

// the batch as a persistent, lane-refilling solve (kc_implicit_sm.cuh)
struct ImpBatchSrc {
  const double* geom23;
  const double* dt;
  double* pp_io;
  int* res;
  __device__ bool load(long i, ImpLane& L) {
    geom_from_record23(geom23 + i * 23, L.g);
    for (int k = 0; k < NV; ++k) L.pp00[k] = pp_io[i * NV + k];
    L.dt = dt[i];
    L.cell = i;
    return true;
  }
  __device__ void store(const ImpLane& L) {
    long i = L.cell;
    int* o = res + i * 6;
    if (L.ok) {
      for (int k = 0; k < NV; ++k) pp_io[i * NV + k] = L.pp[k];
      o[0] = 1;
      o[1] = L.rung;
      o[2] = L.iters;
      o[3] = L.p;
      o[4] = L.e;
      o[5] = L.fr;
    } else {
      o[0] = 0;
      o[1] = -1;
      o[2] = 0;
      o[3] = PRIM_RAD;
      o[4] = EQ_ENERGY;
      o[5] = FRAME_LAB;
    }
  }
};
__global__ void __launch_bounds__(128) k_implicit_batch_persistent(long n, const double* geom23, const double* dt,
                                                                   double* pp_io, int* res, BatchArgs a,
                                                                   unsigned long long* counter) {
  ImpBatchSrc src{geom23, dt, pp_io, res};
  ImpParams P{a.gam, a.rp, a.op, a.ip};
  imp_persistent(src, n, counter, P);
}
// Sort key of a batch cell for the sorted form: the start fluid of the solve
// (the ladder's first branch), then the cell's optical-depth proxy log10(rho dt)
// and its temperature proxy log10(u / rho), each quantised to 1/8 decade, so
// that a warp's lanes get cells that take similar paths through the solver.
__global__ void k_batch_key(long n, const double* __restrict__ geom23, const double* __restrict__ dt,
                            const double* __restrict__ pp_in, BatchArgs a, unsigned* key, int* idx) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  geom_from_record23(geom23 + i * 23, g);
  double pp[NV];
  for (int k = 0; k < NV; ++k) pp[k] = pp_in[i * NV + k];
  double ehat = -calc_ff_rtt(pp, g, nullptr);
  unsigned start = (ehat < a.ip.threshold * pp[UU]) ? 1u : 0u;
  auto q = [](double x, double lo) -> unsigned {  // 1/8-decade bins over 128 decades
    double b = (::log10(x) - lo) * 8.0;
    return (b > 0.0 && b < 1023.0) ? (unsigned)b : (b >= 1023.0 ? 1023u : 0u);
  };
  key[i] = (start << 20) | (q(pp[RHO] * dt[i], -64.0) << 10) | q(pp[UU] / pp[RHO], -64.0);
  idx[i] = (int)i;
}
// launch either form of the batch on `st`; the persistent and sorted forms take
// their scratch from the stream-ordered allocator
int launch_batch(long n, const double* g, const double* d, double* p, int* r, const BatchArgs& a, int mode,
                 cudaStream_t st) {
  if (mode == KC_IMPLICIT_PER_CELL) {
    k_implicit_batch<<<nblk(n), TPB, 0, st>>>(n, g, d, p, r, a);
    return cudaGetLastError() == cudaSuccess ? KC_OK : KC_ERR_CUDA;
  }
  if (mode == KC_IMPLICIT_SORTED) {
    if (n > 0x7fffffffL) return KC_ERR_INVALID_CONFIG;
    unsigned *k0 = nullptr, *k1 = nullptr;
    int *i0 = nullptr, *i1 = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k0, k1, i0, i1, (int)n, 0, 21, st);
    if (cudaMallocAsync((void**)&k0, n * 4, st) != cudaSuccess || cudaMallocAsync((void**)&k1, n * 4, st) != cudaSuccess ||
        cudaMallocAsync((void**)&i0, n * 4, st) != cudaSuccess || cudaMallocAsync((void**)&i1, n * 4, st) != cudaSuccess ||
        cudaMallocAsync(&tmp, tmp_bytes, st) != cudaSuccess)
      return KC_ERR_OOM;
    k_batch_key<<<nblk(n), TPB, 0, st>>>(n, g, d, p, a, k0, i0);
    cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0, k1, i0, i1, (int)n, 0, 21, st);
    k_implicit_batch<<<nblk(n), TPB, 0, st>>>(n, g, d, p, r, a, i1);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(tmp, st);
    cudaFreeAsync(k0, st);
    cudaFreeAsync(k1, st);
    cudaFreeAsync(i0, st);
    cudaFreeAsync(i1, st);
    return e == cudaSuccess ? KC_OK : KC_ERR_CUDA;
  }
  if (mode != KC_IMPLICIT_COMPACTING) return KC_ERR_INVALID_CONFIG;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_implicit_batch_persistent, TPB, 0);
  long need = (n + TPB - 1) / TPB, cap = (long)(per_sm > 0 ? per_sm : 1) * (nsm > 0 ? nsm : 1);
  void* counter = nullptr;
  if (cudaMallocAsync(&counter, sizeof(unsigned long long), st) != cudaSuccess) return KC_ERR_OOM;
  cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
  k_implicit_batch_persistent<<<(unsigned)(need < cap ? need : cap), TPB, 0, st>>>(n, g, d, p, r, a,
                                                                                   (unsigned long long*)counter);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(counter, st);
  return e == cudaSuccess ? KC_OK : KC_ERR_CUDA;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
int batch_prepare(const kc_options* opt, BatchArgs& a) {
  if (!opt || opt->abi_version != KC_ABI_VERSION) return KC_ERR_INVALID_CONFIG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return KC_ERR_NO_DEVICE;
  if (cudaSetDevice(opt->device) != cudaSuccess) return KC_ERR_CUDA;
  SimParams sp;
  params_from_options(*opt, sp);
  a.gam = sp.gam;
  a.rp = sp.rp;
  a.op = sp.op;
  a.ip = sp.ip;
  a.fl = sp.fl;
  return KC_OK;
}

}  // namespace

extern "C" int kc_implicit_batch(const kc_options* opt, int64_t n, const double* geom23, const double* dt, double* pp,
                                 int32_t* res, int32_t mode) {
  BatchArgs a;
  int st = batch_prepare(opt, a);
  if (st) return st;
  if (mode != KC_IMPLICIT_PER_CELL && mode != KC_IMPLICIT_COMPACTING && mode != KC_IMPLICIT_SORTED)
    return KC_ERR_INVALID_CONFIG;
  if (n <= 0) return KC_OK;
  DevBuf dg, dd, dp, dr;
  if (cudaMalloc(&dg.p, n * 23 * 8) || cudaMalloc(&dd.p, n * 8) || cudaMalloc(&dp.p, n * NV * 8) ||
      cudaMalloc(&dr.p, n * 6 * 4))
    return KC_ERR_OOM;
  cudaMemcpy(dg.p, geom23, n * 23 * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dd.p, dt, n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dp.p, pp, n * NV * 8, cudaMemcpyHostToDevice);
  if ((st = launch_batch(n, (const double*)dg.p, (const double*)dd.p, (double*)dp.p, (int*)dr.p, a, mode, 0)))
    return st;
  if (cudaDeviceSynchronize() != cudaSuccess) return KC_ERR_CUDA;
  cudaMemcpy(pp, dp.p, n * NV * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(res, dr.p, n * 6 * 4, cudaMemcpyDeviceToHost);
  return KC_OK;
}

extern "C" int kc_implicit_batch_device(const kc_options* opt, int64_t n, const double* geom23, const double* dt,
                                        double* pp, int32_t* res, int32_t mode, void* stream) {
  BatchArgs a;
  int st = batch_prepare(opt, a);
  if (st) return st;
  if (n <= 0) return KC_OK;
  if (!geom23 || !dt || !pp || !res) return KC_ERR_INVALID_CONFIG;
  return launch_batch(n, geom23, dt, pp, res, a, mode, (cudaStream_t)stream);
}

namespace {
// xorshift64* (the generator family of the reference's implicit battery)
struct XorShift {
  uint64_t s;
  double next() {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return (double)((s * 0x2545F4914F6CDD1DULL) >> 11) * 0x1.0p-53;
  }
  double pm() { return 2.0 * next() - 1.0; }
  double loguni(double lo, double hi) { return kmath::exp(kmath::log(lo) + (kmath::log(hi) - kmath::log(lo)) * next()); }
};
// a spatial 3-velocity (VELR) of Lorentz factor gamma relative to the normal
// observer, in a random direction
void velr_with_gamma(XorShift& rng, const Geom& g, double gamma, double v[3]) {
  double nn[3] = {rng.pm(), rng.pm(), rng.pm()};
  double q = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) q += nn[i] * nn[j] * g.gg[i + 1][j + 1];
  double sc = kmath::sqrt((gamma * gamma - 1.0) / q);
  for (int i = 0; i < 3; ++i) v[i] = nn[i] * sc;
}
}  // namespace

extern "C" int kc_synth_implicit_cells(const kc_options* opt, int64_t n, uint64_t seed, double* geom23, double* dt,
                                       double* pp) {
  if (!opt || opt->abi_version != KC_ABI_VERSION || n < 0 || !geom23 || !dt || !pp) return KC_ERR_INVALID_CONFIG;
  SimParams sp;
  params_from_options(*opt, sp);
  const Consts& con = sp.op.c;
  const long nchunk = 4096;
  host_par(0, (n + nchunk - 1) / nchunk, [&](long k) {
    XorShift rng{seed ^ (0x9E3779B97F4A7C15ULL * (uint64_t)(k + 1))};
    for (long c = k * nchunk; c < n && c < (k + 1) * nchunk; ++c) {
      double r = rng.loguni(3.0, 50.0);
      double th = 0.3 + (KP_PI - 0.6) * rng.next();
      double x[4] = {0.0, kmath::log(r - sp.mp.mksr0), mks2_x2_from_theta(th, sp.mp.mksh0), 0.0};
      Geom g;
      geometry_at(MKS2, sp.mp, x, g);
      double* gr = geom23 + c * 23;
      int q = 0;
      for (int i = 0; i < 4; ++i)
        for (int j = i; j < 4; ++j) {
          gr[q] = g.gg[i][j];
          gr[10 + q] = g.GG[i][j];
          ++q;
        }
      gr[20] = g.gdet;
      gr[21] = g.alpha;
      gr[22] = g.gttpert;
      double* p = pp + c * NV;
      double rho = rng.loguni(1.0e-8, 1.0);
      double tgas = rng.loguni(1.0e5, 1.0e9);
      double ugas = u_from_trho(con, tgas, rho, sp.gam);
      double v[3];
      velr_with_gamma(rng, g, 1.0 / kmath::sqrt(1.0 - 0.81 * rng.next()), v);  // |v| < 0.9c
      p[RHO] = rho;
      p[UU] = ugas;
      p[VX] = v[0];
      p[VY] = v[1];
      p[VZ] = v[2];
      p[ENTR] = s_from_u(rho, ugas, sp.gam);
      double beta = rng.loguni(1.0, 1.0e3);
      double bsq = 2.0 * (sp.gam - 1.0) * ugas / beta;
      velr_with_gamma(rng, g, kmath::sqrt(1.0 + bsq), v);
      p[B1] = v[0];
      p[B2] = v[1];
      p[B3] = v[2];
      p[EE] = ugas / rng.loguni(1.0e-4, 1.0e4);  // E_gas / E_rad log-uniform in [1e-4, 1e4]
      velr_with_gamma(rng, g, 1.0 + rng.next(), v);
      p[FX] = v[0];
      p[FY] = v[1];
      p[FZ] = v[2];
      dt[c] = rng.loguni(1.0e-10, 1.0);
    }
  });
  return KC_OK;
}

extern "C" int kc_u2p_batch(const kc_options* opt, int64_t n, const double* geom23, const double* uu, double* pp,
                            int32_t* flags_out) {
  BatchArgs a;
  int st = batch_prepare(opt, a);
  if (st) return st;
  if (n <= 0) return KC_OK;
  DevBuf dg, du, dp, df;
  if (cudaMalloc(&dg.p, n * 23 * 8) || cudaMalloc(&du.p, n * NV * 8) || cudaMalloc(&dp.p, n * NV * 8) ||
      cudaMalloc(&df.p, n * 3 * 4))
    return KC_ERR_OOM;
  cudaMemcpy(dg.p, geom23, n * 23 * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(du.p, uu, n * NV * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dp.p, pp, n * NV * 8, cudaMemcpyHostToDevice);
  k_u2p_batch<<<nblk(n), TPB>>>(n, (const double*)dg.p, (const double*)du.p, (double*)dp.p, (int*)df.p, a);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return KC_ERR_CUDA;
  cudaMemcpy(pp, dp.p, n * NV * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(flags_out, df.p, n * 3 * 4, cudaMemcpyDeviceToHost);
  return KC_OK;
}

// ==== allocation-free implicit batch ==========================================
// kc_implicit_batch stages the caller's host arrays through device buffers it
// allocates per call. This variant stages them through one fixed, file-scope
// device array instead and allocates nothing: 16384 cells of geometry (23 f64),
// dt (1 f64), primitives (13 f64) and results (6 i32), 5 MiB, held by every
// device that loads the library until the process exits. The address of the
// array on a device is looked up once, with that device current, on the first
// call on that device (that first call should come before any stream capture).
// All calls on a device share the array and leave the last call's contents in
// it; calls that overlap on the same device race on it.
namespace {

const size_t kNoAllocGeomOff = 0;
const size_t kNoAllocDtOff = kNoAllocGeomOff + (size_t)KC_NOALLOC_MAX_CELLS * 23 * 8;
const size_t kNoAllocPpOff = kNoAllocDtOff + (size_t)KC_NOALLOC_MAX_CELLS * 8;
const size_t kNoAllocResOff = kNoAllocPpOff + (size_t)KC_NOALLOC_MAX_CELLS * NV * 8;
const size_t kNoAllocBytes = kNoAllocResOff + (size_t)KC_NOALLOC_MAX_CELLS * 6 * 4;
static_assert(kNoAllocDtOff % 256 == 0 && kNoAllocPpOff % 256 == 0 && kNoAllocResOff % 256 == 0,
              "scratch regions stay 256-byte aligned");

// host-side stand-in for the device array; its device address comes from
// cudaGetSymbolAddress
static __device__ __align__(256) unsigned char kc_noalloc_scratch[kNoAllocBytes];

const int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// the scratch array's address on the current device (set-up on first use)
int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return KC_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, kc_noalloc_scratch) != cudaSuccess || !ptr) return KC_ERR_CUDA;
    g_noalloc_ptr[dev] = (unsigned char*)ptr;
  }
  *out = g_noalloc_ptr[dev];
  return KC_OK;
}

}  // namespace

extern "C" int kc_implicit_batch_noalloc(const kc_options* opt, int64_t n, const double* geom23, const double* dt,
                                         double* pp, int32_t* res, int32_t mode) {
  if (n > KC_NOALLOC_MAX_CELLS) return KC_ERR_TOO_MANY_CELLS;
  BatchArgs a;
  int st = batch_prepare(opt, a);
  if (st) return st;
  if (mode != KC_IMPLICIT_PER_CELL) return KC_ERR_INVALID_CONFIG;
  if (n <= 0) return KC_OK;
  if (!geom23 || !dt || !pp || !res) return KC_ERR_INVALID_CONFIG;
  unsigned char* base = nullptr;
  if ((st = noalloc_scratch(&base))) return st;
  double* dg = (double*)(base + kNoAllocGeomOff);
  double* dd = (double*)(base + kNoAllocDtOff);
  double* dp = (double*)(base + kNoAllocPpOff);
  int* dr = (int*)(base + kNoAllocResOff);
  // every result entry of the n cells is written by the kernel; cleared anyway so
  // that nothing of an earlier call can be read back
  if (cudaMemset(dr, 0, (size_t)n * 6 * 4) != cudaSuccess ||
      cudaMemcpy(dg, geom23, (size_t)n * 23 * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dd, dt, (size_t)n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dp, pp, (size_t)n * NV * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    return KC_ERR_CUDA;
  k_implicit_batch<<<nblk(n), TPB>>>(n, dg, dd, dp, dr, a);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return KC_ERR_CUDA;
  if (cudaMemcpy(pp, dp, (size_t)n * NV * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(res, dr, (size_t)n * 6 * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return KC_ERR_CUDA;
  return KC_OK;
}

// ---- the learned-guess network: training, forward and gradient entry points --
namespace {
static_assert(MLP_NW == KC_MLP_NWEIGHTS, "weight blob size");
// minibatch indices of one training step: splitmix64 of (seed, step, slot)
__global__ void k_mlp_sample(long* idx, long nb, long n, uint64_t seed, long step) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t)(step * nb + i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  idx[i] = (long)(z % (uint64_t)n);
}
const int MLP_ACT = MLP_IN + 4 * MLP_H + MLP_OUT;  // per-sample training record (floats)
int mlp_device() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return KC_ERR_NO_DEVICE;
  return KC_OK;
}
}  // namespace

extern "C" int kc_mlp_forward(const float* weights, int64_t n, const float* features_std, float* out_std) {
  int st = mlp_device();
  if (st) return st;
  if (!weights || n < 0 || (n > 0 && (!features_std || !out_std))) return KC_ERR_INVALID_CONFIG;
  if (n == 0) return KC_OK;
  DevBuf db, dw1, dw2, dw3, dx, dy;
  if (cudaMalloc(&db.p, MLP_NW * 4) || cudaMalloc(&dw1.p, MLP_H * MLP_IN * 2) || cudaMalloc(&dw2.p, MLP_H * MLP_H * 2) ||
      cudaMalloc(&dw3.p, 8 * MLP_H * 2) || cudaMalloc(&dx.p, n * MLP_IN * 4) || cudaMalloc(&dy.p, n * MLP_OUT * 4))
    return KC_ERR_OOM;
  cudaMemcpy(db.p, weights, MLP_NW * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dx.p, features_std, n * MLP_IN * 4, cudaMemcpyHostToDevice);
  k_mlp_pack<<<(MLP_H * MLP_H + 127) / 128, 128>>>((const float*)db.p, (__nv_bfloat16*)dw1.p, (__nv_bfloat16*)dw2.p,
                                                   (__nv_bfloat16*)dw3.p);
  MlpDev m = {(const __nv_bfloat16*)dw1.p, (const __nv_bfloat16*)dw2.p, (const __nv_bfloat16*)dw3.p,
              (const float*)db.p};
  k_mlp_forward<<<nblk(n), TPB>>>(m, n, (const float*)dx.p, (float*)dy.p);
  if (cudaDeviceSynchronize() != cudaSuccess) return KC_ERR_CUDA;
  cudaMemcpy(out_std, dy.p, n * MLP_OUT * 4, cudaMemcpyDeviceToHost);
  return KC_OK;
}

extern "C" int kc_mlp_grad(const float* weights, int64_t n, const float* features_std, const float* targets_std,
                           float* grad, float* loss) {
  int st = mlp_device();
  if (st) return st;
  if (!weights || !grad || !loss || n <= 0 || !features_std || !targets_std) return KC_ERR_INVALID_CONFIG;
  DevBuf db, dx, dt, da, dg, dl;
  if (cudaMalloc(&db.p, MLP_NW * 4) || cudaMalloc(&dx.p, n * MLP_IN * 4) || cudaMalloc(&dt.p, n * MLP_OUT * 4) ||
      cudaMalloc(&da.p, n * MLP_ACT * 4) || cudaMalloc(&dg.p, MLP_NW * 4) || cudaMalloc(&dl.p, 4))
    return KC_ERR_OOM;
  cudaMemcpy(db.p, weights, MLP_NW * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dx.p, features_std, n * MLP_IN * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dt.p, targets_std, n * MLP_OUT * 4, cudaMemcpyHostToDevice);
  cudaMemset(dg.p, 0, MLP_NW * 4);
  cudaMemset(dl.p, 0, 4);
  k_mlp_train_fwd<<<nblk(n), TPB>>>((const float*)db.p, (const float*)dx.p, (const float*)dt.p, nullptr, n,
                                    (float*)da.p, (float*)dl.p);
  k_mlp_train_grad<<<(MLP_NW + 127) / 128, 128>>>((const float*)da.p, n, (float*)dg.p);
  if (cudaDeviceSynchronize() != cudaSuccess) return KC_ERR_CUDA;
  cudaMemcpy(grad, dg.p, MLP_NW * 4, cudaMemcpyDeviceToHost);
  float l = 0.0f;
  cudaMemcpy(&l, dl.p, 4, cudaMemcpyDeviceToHost);
  *loss = l / (float)(n * MLP_OUT);
  return KC_OK;
}

// Training: the normalisation (per-column mean and standard deviation) is
// taken from the pairs on the host, the feature deviations floored at
// MLP_FEATURE_STD_MIN and the standardised features clipped to
// +-MLP_STD_CLIP as inference clips them; the weights start He-uniform
// from `seed` (biases zero); each step draws `batch` pairs, runs the forward
// and backward kernels and an Adam update with learning rate `lr`.
extern "C" int kc_mlp_train(const float* features, const float* targets, int64_t n, int32_t steps, int32_t batch,
                            float lr, uint64_t seed, float* weights_out, float* loss_curve) {
  int st = mlp_device();
  if (st) return st;
  if (!features || !targets || !weights_out || n <= 0 || steps < 0 || batch <= 0 || !(lr > 0.0f))
    return KC_ERR_INVALID_CONFIG;
  std::vector<float> w(MLP_NW, 0.0f), xs((size_t)n * MLP_IN), ts((size_t)n * MLP_OUT);
  auto standardise = [&](const float* src, int cols, int off_mean, int off_std, double floor, double clip,
                         float* dst) {
    for (int k = 0; k < cols; ++k) {
      double s = 0.0, q = 0.0;
      for (int64_t i = 0; i < n; ++i) s += src[i * cols + k];
      double mu = s / (double)n;
      for (int64_t i = 0; i < n; ++i) q += (src[i * cols + k] - mu) * (src[i * cols + k] - mu);
      double sd = std::sqrt(q / (double)n);
      if (!(sd > floor)) sd = floor;
      w[off_mean + k] = (float)mu;
      w[off_std + k] = (float)sd;
      for (int64_t i = 0; i < n; ++i) {
        double z = ((double)src[i * cols + k] - (double)w[off_mean + k]) / (double)w[off_std + k];
        dst[i * cols + k] = (float)(z > clip ? clip : (z < -clip ? -clip : z));
      }
    }
  };
  standardise(features, MLP_IN, MLP_OFF_IMEAN, MLP_OFF_ISTD, MLP_FEATURE_STD_MIN, MLP_STD_CLIP, xs.data());
  standardise(targets, MLP_OUT, MLP_OFF_OMEAN, MLP_OFF_OSTD, 1.0e-30, 1.0e30, ts.data());
  for (float v : xs)
    if (!std::isfinite(v)) return KC_ERR_INVALID_CONFIG;
  for (float v : ts)
    if (!std::isfinite(v)) return KC_ERR_INVALID_CONFIG;
  XorShift rng{seed ? seed : 0x2545F4914F6CDD1DULL};
  auto he = [&](int off, int rows, int cols) {
    double a = std::sqrt(6.0 / cols);
    for (int i = 0; i < rows * cols; ++i) w[off + i] = (float)(a * rng.pm());
  };
  he(MLP_OFF_W1, MLP_H, MLP_IN);
  he(MLP_OFF_W2, MLP_H, MLP_H);
  he(MLP_OFF_W3, MLP_OUT, MLP_H);
  long nb = batch < n ? batch : n;
  DevBuf db, dg, dm1, dm2, dx, dt, di, da, dl;
  if (cudaMalloc(&db.p, MLP_NW * 4) || cudaMalloc(&dg.p, MLP_NW * 4) || cudaMalloc(&dm1.p, MLP_NW * 4) ||
      cudaMalloc(&dm2.p, MLP_NW * 4) || cudaMalloc(&dx.p, n * MLP_IN * 4) || cudaMalloc(&dt.p, n * MLP_OUT * 4) ||
      cudaMalloc(&di.p, nb * 8) || cudaMalloc(&da.p, nb * MLP_ACT * 4) || cudaMalloc(&dl.p, (steps + 1) * 4))
    return KC_ERR_OOM;
  cudaMemcpy(db.p, w.data(), MLP_NW * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dx.p, xs.data(), n * MLP_IN * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dt.p, ts.data(), n * MLP_OUT * 4, cudaMemcpyHostToDevice);
  cudaMemset(dm1.p, 0, MLP_NW * 4);
  cudaMemset(dm2.p, 0, MLP_NW * 4);
  cudaMemset(dl.p, 0, (steps + 1) * 4);
  double b1 = 1.0, b2 = 1.0;
  for (int s = 0; s < steps; ++s) {
    b1 *= 0.9;
    b2 *= 0.999;
    k_mlp_sample<<<nblk(nb), TPB>>>((long*)di.p, nb, n, seed, s);
    k_mlp_train_fwd<<<nblk(nb), TPB>>>((const float*)db.p, (const float*)dx.p, (const float*)dt.p,
                                       (const long*)di.p, nb, (float*)da.p, (float*)dl.p + s);
    k_mlp_train_grad<<<(MLP_NW + 127) / 128, 128>>>((const float*)da.p, nb, (float*)dg.p);
    k_mlp_adam<<<(MLP_NW + 127) / 128, 128>>>((float*)db.p, (const float*)dg.p, (float*)dm1.p, (float*)dm2.p, lr,
                                              (float)(1.0 - b1), (float)(1.0 - b2));
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return KC_ERR_CUDA;
  cudaMemcpy(weights_out, db.p, MLP_NW * 4, cudaMemcpyDeviceToHost);
  if (loss_curve && steps > 0) {
    std::vector<float> l(steps);
    cudaMemcpy(l.data(), dl.p, steps * 4, cudaMemcpyDeviceToHost);
    for (int s = 0; s < steps; ++s) loss_curve[s] = l[s] / (float)(nb * MLP_OUT);
  }
  return KC_OK;
}

// ---- FP64 pipe peak: a DFMA-chain microbenchmark (the FP64 roofline) -------------
namespace {
const int DFMA_CHAINS = 16;
__global__ void __launch_bounds__(256) k_dfma_chains(double* sink, int iters, double b, double c) {
  double a[DFMA_CHAINS];
  for (int k = 0; k < DFMA_CHAINS; ++k) a[k] = 1.0e-3 * (threadIdx.x + k);
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < DFMA_CHAINS; ++k) a[k] = __fma_rn(a[k], b, c);
  double s = 0.0;
  for (int k = 0; k < DFMA_CHAINS; ++k) s += a[k];
  if (s == -1.0) sink[blockIdx.x] = s;  // never true; keeps the chains live
}
}  // namespace

// Best of five launches of independent DFMA chains over every SM, in TFLOP/s
// (2 FLOP per DFMA). Runs on the current device.
extern "C" int kc_fp64_peak(double* tflops) {
  int st = mlp_device();
  if (st) return st;
  if (!tflops) return KC_ERR_INVALID_CONFIG;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = nsm * 8, threads = 256, iters = 1 << 14;
  DevBuf sink;
  if (cudaMalloc(&sink.p, (size_t)blocks * 8)) return KC_ERR_OOM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_dfma_chains<<<blocks, threads>>>((double*)sink.p, 256, 0.999999, 1.0e-7);
  float best = 1.0e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    k_dfma_chains<<<blocks, threads>>>((double*)sink.p, iters, 0.999999, 1.0e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess) return KC_ERR_CUDA;
  *tflops = 2.0 * DFMA_CHAINS * (double)iters * blocks * threads / (best * 1.0e-3) / 1.0e12;
  return KC_OK;
}

// ---- autotuner -------------------------------------------------------------------
namespace {
struct TuneConfig {
  int implicit_mode, tpb_implicit, tpb_flux, tpb_u2p, phi_fastest;
};
void tune_apply(kc_handle* h, const TuneConfig& c) {
  h->opt.implicit_mode = c.implicit_mode;
  h->implicit_phi_fastest = c.phi_fastest;
  h->tpb_implicit = c.tpb_implicit;
  h->tpb_flux = c.tpb_flux;
  h->tpb_u2p = c.tpb_u2p;
  drop_graph(h);
}
TuneConfig tune_current(const kc_handle* h) {
  return {h->opt.implicit_mode, h->tpb_implicit, h->tpb_flux, h->tpb_u2p, h->implicit_phi_fastest};
}
// The state a step reads and writes across steps: p, u, flags on the device and
// the handle's step scalars and counters.
struct TuneSnapshot {
  double *p = nullptr, *u = nullptr;
  int* flags = nullptr;
  kc_counters c;
  long long n_launch = 0;
};
void tune_save(kc_handle* h, TuneSnapshot& sn) {
  size_t nb = (size_t)NV * h->gr.nc * 8;
  cudaMemcpyAsync(sn.p, h->ds.p, nb, cudaMemcpyDeviceToDevice, h->stream);
  cudaMemcpyAsync(sn.u, h->ds.u, nb, cudaMemcpyDeviceToDevice, h->stream);
  cudaMemcpyAsync(sn.flags, h->ds.flags, (size_t)6 * h->gr.nc * 4, cudaMemcpyDeviceToDevice, h->stream);
  kc_get_counters(h, &sn.c);
  sn.n_launch = h->n_launch;
}
void tune_restore(kc_handle* h, const TuneSnapshot& sn) {
  size_t nb = (size_t)NV * h->gr.nc * 8;
  cudaMemcpyAsync(h->ds.p, sn.p, nb, cudaMemcpyDeviceToDevice, h->stream);
  cudaMemcpyAsync(h->ds.u, sn.u, nb, cudaMemcpyDeviceToDevice, h->stream);
  cudaMemcpyAsync(h->ds.flags, sn.flags, (size_t)6 * h->gr.nc * 4, cudaMemcpyDeviceToDevice, h->stream);
  kc_set_counters(h, &sn.c);
  h->n_launch = sn.n_launch;
}
}  // namespace

// Picks the implicit form (per-cell or split), the block sizes of the
// per-cell implicit, face-flux and u2p kernels and the per-cell implicit
// kernel's cell order (phi on 3D or theta on 2D fastest, or x fastest) by
// timing whole steps on the
// handle's current state, one knob at a time (coordinate descent from the
// configuration on entry). Each trial restores the state, runs one untimed step
// (with the graph form on, a second one, so the timed steps replay the graph)
// and times `steps` steps with CUDA events on the handle's stream. Every
// candidate gives bit-identical results, so the choice changes speed only. The
// state and counters are restored at the end, and the best configuration stays
// set. The learned guess and the harvest keep their fixed forms (not tuned
// while either is on).
extern "C" int kc_autotune(kc_handle* h, int32_t steps, kc_tune_result* out) {
  if (!h || steps < 1) return KC_ERR_INVALID_CONFIG;
  if (h->last_status) return h->last_status;
  if (h->guess_mode != KC_GUESS_PLAIN || h->hcap > 0)
    return reject(h, KC_ERR_INVALID_CONFIG, "autotune with the learned guess or the harvest on");
  if (h->timing) return reject(h, KC_ERR_INVALID_CONFIG, "autotune with pass timing on");
  int st = cuda_check(h, cudaStreamSynchronize(h->stream), "autotune");
  if (st) return st;
  TuneSnapshot sn;
  size_t nb = (size_t)NV * h->gr.nc * 8;
  if (cudaMalloc(&sn.p, nb) || cudaMalloc(&sn.u, nb) || cudaMalloc(&sn.flags, (size_t)6 * h->gr.nc * 4)) {
    cudaFree(sn.p);
    cudaFree(sn.u);
    cudaFree(sn.flags);
    return fail(h, KC_ERR_OOM, "autotune snapshot");
  }
  tune_save(h, sn);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int trials = 0;
  auto measure = [&](const TuneConfig& c, double& ms) -> int {
    tune_restore(h, sn);
    tune_apply(h, c);
    int warm = h->use_graph ? 2 : 1;
    for (int k = 0; k < warm; ++k)
      if (int r = run_step(h, NAN, nullptr)) return r;
    cudaEventRecord(e0, h->stream);
    for (int k = 0; k < steps; ++k)
      if (int r = run_step(h, NAN, nullptr)) return r;
    cudaEventRecord(e1, h->stream);
    cudaEventSynchronize(e1);
    float f = 0.0f;
    cudaEventElapsedTime(&f, e0, e1);
    ms = f / steps;
    ++trials;
    return KC_OK;
  };
  TuneConfig best = tune_current(h), entry = best;
  double best_ms = 0.0, entry_ms = 0.0;
  st = measure(best, best_ms);
  entry_ms = best_ms;
  const int forms[2] = {KC_IMPLICIT_PER_CELL, KC_IMPLICIT_SPLIT};
  const int sizes[3] = {64, 96, 128};
  for (int knob = 0; knob < 5 && !st; ++knob) {
    int n = (knob == 0 || knob == 4) ? 2 : 3;
    for (int i = 0; i < n && !st; ++i) {
      TuneConfig c = best;
      if (knob == 0) c.implicit_mode = forms[i];
      if (knob == 1) c.tpb_implicit = sizes[i];
      if (knob == 2) c.tpb_flux = sizes[i];
      if (knob == 3) c.tpb_u2p = sizes[i];
      if (knob == 4) c.phi_fastest = i;
      if (memcmp(&c, &best, sizeof c) == 0) continue;
      double ms = 0.0;
      st = measure(c, ms);
      if (!st && ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
  }
  tune_restore(h, sn);
  tune_apply(h, st ? entry : best);
  cudaStreamSynchronize(h->stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sn.p);
  cudaFree(sn.u);
  cudaFree(sn.flags);
  if (st) return st;
  if (out) {
    out->implicit_mode = best.implicit_mode;
    out->tpb_implicit = best.tpb_implicit;
    out->tpb_flux = best.tpb_flux;
    out->tpb_u2p = best.tpb_u2p;
    out->implicit_phi_fastest = best.phi_fastest;
    out->ms_per_step = best_ms;
    out->ms_per_step_entry = entry_ms;
    out->trials = trials;
  }
  return KC_OK;
}

// ---- KDMP v2 checkpoints (koral/io/dump.zig) ---------------------------------------
extern "C" int kc_kdmp_write_header(const kc_dump_header* hd, uint8_t* out) {
  if (!hd || !out) return KC_ERR_INVALID_CONFIG;
  kdump::write_header(*hd, out);
  return KC_OK;
}
extern "C" int kc_kdmp_parse_header(const uint8_t* bytes, int64_t len, kc_dump_header* hd) {
  if (!hd) return KC_ERR_INVALID_CONFIG;
  return kdump::parse_header(bytes, len, *hd);
}
extern "C" int64_t kc_kdmp_size(kc_handle* h) {
  if (!h) return -1;
  return KC_KDMP_HEADER_SIZE + kdump::body_bytes(h->gr.nx, h->gr.ny, h->gr.nz, NV);
}
extern "C" int kc_kdmp_write(kc_handle* h, uint32_t out_idx, uint8_t* out, int64_t capacity, int64_t* written) {
  if (!h || !out) return KC_ERR_INVALID_CONFIG;
  if (written) *written = 0;
  int64_t need = kc_kdmp_size(h);
  if (capacity < need) return reject(h, KC_ERR_INVALID_CONFIG, "KDMP buffer smaller than kc_kdmp_size");
  const DGrid& gr = h->gr;
  long nd = (long)gr.nx * gr.ny * gr.nz;
  // the staging array holds NV x (cells incl. ghosts) doubles, more than the body
  k_domain_to_kdmp<<<nblk(nd * NV, 256), 256, 0, h->stream>>>(h->ds, h->staging);
  int st = cuda_check(h, cudaMemcpyAsync(out + KC_KDMP_HEADER_SIZE, h->staging, (size_t)nd * NV * 8,
                                         cudaMemcpyDeviceToHost, h->stream), "KDMP write");
  if (!st) st = cuda_check(h, cudaStreamSynchronize(h->stream), "KDMP write");
  if (st) return st;
  kc_dump_header hd = {(uint32_t)gr.nx, (uint32_t)gr.ny, (uint32_t)gr.nz, (uint32_t)NV, h->t, (uint64_t)h->nstep,
                       out_idx};
  kdump::write_header(hd, out);
  if (written) *written = need;
  return KC_OK;
}
extern "C" int kc_kdmp_load(kc_handle* h, const uint8_t* bytes, int64_t len, kc_dump_header* hd_out) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  kc_dump_header hd;
  int st = kdump::parse_header(bytes, len, hd);
  if (st) return reject(h, st, "KDMP header");
  const DGrid& gr = h->gr;
  if (hd.nx != (uint32_t)gr.nx || hd.ny != (uint32_t)gr.ny || hd.nz != (uint32_t)gr.nz || hd.nv != (uint32_t)NV)
    return reject(h, KC_ERR_KDMP_DIM_MISMATCH, "KDMP grid differs from the handle's");
  long nd = (long)gr.nx * gr.ny * gr.nz;
  if (len < kc_kdmp_size(h)) return reject(h, KC_ERR_KDMP_TRUNCATED, "KDMP body truncated");
  st = cuda_check(h, cudaMemcpyAsync(h->staging, bytes + KC_KDMP_HEADER_SIZE, (size_t)nd * NV * 8,
                                     cudaMemcpyHostToDevice, h->stream), "KDMP load");
  if (st) return st;
  k_kdmp_to_domain<<<nblk(nd), TPB, 0, h->stream>>>(h->ds, h->staging, h->sp.gam);
  st = cuda_check(h, cudaStreamSynchronize(h->stream), "KDMP load");
  if (st) return st;
  if (hd_out) *hd_out = hd;
  return KC_OK;
}
extern "C" int kc_kdmp_write_file(kc_handle* h, const char* path, uint32_t out_idx) {
  if (!h || !path) return KC_ERR_INVALID_CONFIG;
  int64_t n = kc_kdmp_size(h);
  std::vector<uint8_t> buf((size_t)n);
  int st = kc_kdmp_write(h, out_idx, buf.data(), n, nullptr);
  if (st) return st;
  FILE* f = fopen(path, "wb");
  if (!f) return reject(h, KC_ERR_IO, std::string("cannot create ") + path);
  size_t w = fwrite(buf.data(), 1, buf.size(), f);
  int c = fclose(f);
  if (w != buf.size() || c != 0) return reject(h, KC_ERR_IO, std::string("cannot write ") + path);
  return KC_OK;
}
extern "C" int kc_kdmp_load_file(kc_handle* h, const char* path, kc_dump_header* hd) {
  if (!h || !path) return KC_ERR_INVALID_CONFIG;
  FILE* f = fopen(path, "rb");
  if (!f) return reject(h, KC_ERR_IO, std::string("cannot open ") + path);
  std::vector<uint8_t> buf;
  uint8_t chunk[1 << 16];
  size_t r;
  while ((r = fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + r);
  bool err = ferror(f) != 0;
  fclose(f);
  if (err) return reject(h, KC_ERR_IO, std::string("cannot read ") + path);
  return kc_kdmp_load(h, buf.data(), (int64_t)buf.size(), hd);
}
