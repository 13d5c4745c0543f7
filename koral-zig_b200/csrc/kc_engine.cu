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
  // block sizes of the per-cell implicit, face-flux and u2p kernels (kc_autotune);
  // the implicit kernel's block fills an SM: 256 (255 registers), 384 (168) or
  // 512 threads (128)
  int tpb_implicit = KC_IMPLICIT_TPB, tpb_flux = TPB, tpb_u2p = TPB;
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
  // the y and z face sweeps of the plain form: 0 one thread per face with its own
  // two PPMs, 1 tiles with the reconstructed faces in shared memory, 2 tiles that
  // also stage the stencil rows in shared memory
  int face_tiles = 0;
  // harvest every first-rung converged cell (0), or only those whose pre-solve
  // state fails the Newton core's first residual test (1)
  int harvest_filter = 0;
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
  int fail_alloc_at = 0;  // host-side test hook: the n-th next optional allocation fails (0: none)
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
// An allocation for an optional form (the split implicit buffers, the learned
// guess, the harvest records): on failure nothing is published, the message
// is kept for kc_last_error, the handle stays usable and nullptr is returned.
template <class T>
T* try_dalloc(kc_handle* h, size_t n) {
  if (h->fail_alloc_at > 0 && --h->fail_alloc_at == 0) {
    h->err = "cudaMalloc: out of memory (injected)";
    return nullptr;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T) + 16);
  if (e == cudaSuccess) e = cudaMemset(p, 0, n * sizeof(T) + 16);
  if (e != cudaSuccess) {
    cudaGetLastError();  // an allocation failure is not a device fault: clear it for later checks
    if (p) cudaFree(p);
    h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return nullptr;
  }
  h->allocs.push_back(p);
  return (T*)p;
}
void dfree(kc_handle* h, void* p) {
  if (!p) return;
  for (size_t i = 0; i < h->allocs.size(); ++i)
    if (h->allocs[i] == p) {
      h->allocs.erase(h->allocs.begin() + i);
      break;
    }
  cudaFree(p);
}

// ---- metric cache, built once on the device (koral/metric/precompute.zig:175) ---
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

// The split implicit form's compact list (count, cell indices, warm starts),
// allocated when the form is selected, outside any step and any capture; the
// three pointers are published together or not at all.
int ensure_split(kc_handle* h) {
  if (h->split_count) return KC_OK;
  const DGrid& gr = h->gr;
  long ndom = (long)gr.nx * gr.ny * gr.nz;
  unsigned long long* cnt = try_dalloc<unsigned long long>(h, 1);
  int* cell = cnt ? try_dalloc<int>(h, ndom) : nullptr;
  double* pp0 = cell ? try_dalloc<double>(h, (size_t)NV * ndom) : nullptr;
  if (!pp0) {
    dfree(h, cell);
    dfree(h, cnt);
    return reject(h, KC_ERR_OOM, h->err);
  }
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_implicit_ladder, TPB, 0);
  h->split_blocks = (per_sm > 0 ? per_sm : 1) * (nsm > 0 ? nsm : 1);
  h->split_count = cnt;
  h->split_cell = cell;
  h->split_pp0 = pp0;
  return KC_OK;
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
  // the split form's buffers exist whenever the form is selected (ensure_split)
  if (h->opt.implicit_mode == KC_IMPLICIT_SPLIT && !extra && h->split_count) {
    long ndom = (long)gr.nx * gr.ny * gr.nz;
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
  ImplExtra x = {nullptr, nullptr, nullptr, nullptr, 0, nullptr, 0};
  if (h->imp_ctr) {
    x.n_fallback = h->imp_ctr;
    if (h->hcap > 0) {
      x.hx = h->hx;
      x.ht = h->ht;
      x.hcount = h->imp_ctr + 1;
      x.hcap = h->hcap;
      x.hfilter = h->harvest_filter;
    }
  }
  if (h->guess_mode == KC_GUESS_MLP) {
    MlpDev m = {h->mlp_w1, h->mlp_w2, h->mlp_w3, h->mlp_blob};
    ++h->n_launch;
    k_mlp_guess<<<nblk(ndom), TPB, 0, h->stream>>>(h->ds, m, a, h->guess);
    x.guess = h->guess;
  }
  ++h->n_launch;
  // one block per SM; the learned-guess and harvest forms in the default block
  const int nt = extra || (h->tpb_implicit != 256 && h->tpb_implicit != 512) ? KC_IMPLICIT_TPB : h->tpb_implicit;
  const unsigned nb = nblk(ndom, nt);
  cudaStream_t st = h->stream;
  if (h->hcap > 0) k_implicit<IMPL_FULL, KC_IMPLICIT_TPB><<<nb, nt, 0, st>>>(h->ds, h->dsc, a, x);
  else if (extra) k_implicit<IMPL_GUESS, KC_IMPLICIT_TPB><<<nb, nt, 0, st>>>(h->ds, h->dsc, a, x);
  else if (nt == 256) k_implicit<IMPL_PLAIN, 256><<<nb, nt, 0, st>>>(h->ds, h->dsc, a, x);
  else if (nt == 512) k_implicit<IMPL_PLAIN, 512><<<nb, nt, 0, st>>>(h->ds, h->dsc, a, x);
  else k_implicit<IMPL_PLAIN, KC_IMPLICIT_TPB><<<nb, nt, 0, st>>>(h->ds, h->dsc, a, x);
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

// the FP32 pieces a precision mode selects. KC_MIXED is the set that keeps the
// integrated accretion rate and luminosity of the 192x180x64 wedge within 1e-4
// of plain FP64 after 1000 steps (LAXF 4.5e-10 / 2.4e-7, CT 3.3e-10 / 3.5e-7);
// the FP32 reconstruction alone moves them by 9e-3 / 5.6 and is left out.
int fp32_pieces(int precision) {
  if (precision == KC_MIXED) return KC_FP32_LAXF | KC_FP32_CT;
  return precision & (KC_FP32_PPM | KC_FP32_LAXF | KC_FP32_CT | KC_FP32_FLUX);
}

void launch_face_fluxes(kc_handle* h) {
  const DGrid& gr = h->gr;
  FluxArgs a;
  a.gam = h->sp.gam;
  a.theta = h->sp.minmod_theta;
  a.maxvel = h->sp.maxradviscvel;
  a.fl = h->sp.fl;
  a.radvisc = h->sp.radviscosity;
  a.fp32 = fp32_pieces(h->opt.precision);
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
    bool mx = (a.fp32 & (KC_FP32_PPM | KC_FP32_LAXF | KC_FP32_FLUX)) != 0;
    if (dim == 0) {
      if (mx) k_face_flux<true, 0><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
      else k_face_flux<false, 0><<<nb, tb, 0, h->stream>>>(h->ds, h->dsc, a);
    } else if (!mx && h->face_tiles) {
      // FT_COLS transverse columns x FT_FACES faces per block of 4 warps
      dim3 grid((unsigned)((n0 * n1 + FT_COLS - 1) / FT_COLS), (unsigned)((dims[dim] + 1 + FT_FACES - 1) / FT_FACES));
      const unsigned tb4 = 32 * FT_FACES;
      if (h->face_tiles == 2) {  // stencil rows staged in shared memory
        if (dim == 1) k_face_flux_tiled<1, true><<<grid, tb4, sizeof(FaceTile), h->stream>>>(h->ds, h->dsc, a);
        else k_face_flux_tiled<2, true><<<grid, tb4, sizeof(FaceTile), h->stream>>>(h->ds, h->dsc, a);
      } else {  // stencil through L1, reconstructed faces in shared memory
        if (dim == 1) k_face_flux_tiled<1, false><<<grid, tb4, sizeof(FaceTileOut), h->stream>>>(h->ds, h->dsc, a);
        else k_face_flux_tiled<2, false><<<grid, tb4, sizeof(FaceTileOut), h->stream>>>(h->ds, h->dsc, a);
      }
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
  const bool ct32 = (fp32_pieces(h->opt.precision) & KC_FP32_CT) != 0;
  if (ct32) k_ct_emf<float><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
  else k_ct_emf<double><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
  ++h->n_launch;
  if (ct32) k_ct_rebuild<float><<<nblk(n, 256), 256, 0, h->stream>>>(h->ds);
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
  k_scale_height<<<(unsigned)gr.nx, SH_THREADS, 0, h->stream>>>(h->ds);
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
  // the tiled face kernels stage more than the default 48 KB of shared memory
  st = cuda_check(h, cudaFuncSetAttribute(k_face_flux_tiled<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(FaceTile)), "face tile shared memory");
  if (!st) st = cuda_check(h, cudaFuncSetAttribute(k_face_flux_tiled<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)sizeof(FaceTile)), "face tile shared memory");
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
  if (h->opt.implicit_mode == KC_IMPLICIT_SPLIT && (st = ensure_split(h))) return fail(h, st, h->err);
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
  k_scale_height<<<(unsigned)gr.nx, SH_THREADS, 0, h->stream>>>(ds2);
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

// Test hook: the n-th next optional allocation (split-form buffers, learned
// guess, harvest records, their counters) fails as if the device were out of
// memory, so the OOM paths run without exhausting a shared GPU; 0 disarms.
int kc_debug_fail_allocs(kc_handle* h, int32_t n) {
  if (!h || n < 0) return KC_ERR_INVALID_CONFIG;
  h->fail_alloc_at = n;
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
  const int pieces = KC_FP32_PPM | KC_FP32_LAXF | KC_FP32_CT | KC_FP32_FLUX;
  if (mode != KC_PLAIN_FP64 && mode != KC_MIXED && (mode & ~pieces) != 0)
    return reject(h, KC_ERR_INVALID_CONFIG, "unknown precision mode");
  h->opt.precision = mode;
  drop_graph(h);
  return KC_OK;
}
int kc_set_implicit_mode(kc_handle* h, int32_t mode) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (mode != KC_IMPLICIT_PER_CELL && mode != KC_IMPLICIT_COMPACTING && mode != KC_IMPLICIT_SPLIT)
    return reject(h, KC_ERR_INVALID_CONFIG, "unknown implicit mode");
  if (mode == KC_IMPLICIT_SPLIT) {
    int st = ensure_split(h);
    if (st) return st;  // the form stays as it was
  }
  h->opt.implicit_mode = mode;
  drop_graph(h);
  return KC_OK;
}
static int ensure_imp_ctr(kc_handle* h) {
  if (!h->imp_ctr) h->imp_ctr = try_dalloc<unsigned long long>(h, 2);
  return h->imp_ctr ? KC_OK : reject(h, KC_ERR_OOM, h->err);
}
// The CUDA graph form of the step (no reference counterpart): on, the whole
// step's launch sequence is captured once and replayed (bit-identical).
// The y and z face sweeps' form (no reference counterpart; all bit-identical):
// 0 one thread per face, 1 shared-memory tiles of reconstructed faces, 2 tiles
// that also stage the stencil rows.
int kc_set_face_tiles(kc_handle* h, int32_t mode) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (mode < 0 || mode > 2) return reject(h, KC_ERR_INVALID_CONFIG, "unknown face-tile mode");
  h->face_tiles = mode;
  drop_graph(h);
  return KC_OK;
}
int kc_set_implicit_threads(kc_handle* h, int32_t threads) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (threads != 256 && threads != 384 && threads != 512)
    return reject(h, KC_ERR_INVALID_CONFIG, "implicit threads per block must be 256, 384 or 512");
  h->tpb_implicit = threads;
  drop_graph(h);
  return KC_OK;
}
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
  if (st) return st;
  if (!h->mlp_blob) {  // the five buffers are published together or not at all
    float* blob = try_dalloc<float>(h, MLP_NW);
    __nv_bfloat16* w1 = blob ? try_dalloc<__nv_bfloat16>(h, MLP_H * MLP_IN) : nullptr;
    __nv_bfloat16* w2 = w1 ? try_dalloc<__nv_bfloat16>(h, MLP_H * MLP_H) : nullptr;
    __nv_bfloat16* w3 = w2 ? try_dalloc<__nv_bfloat16>(h, 8 * MLP_H) : nullptr;
    double* guess = w3 ? try_dalloc<double>(h, (size_t)NV * ndom) : nullptr;
    if (!guess) {
      dfree(h, w3);
      dfree(h, w2);
      dfree(h, w1);
      dfree(h, blob);
      return reject(h, KC_ERR_OOM, h->err);
    }
    h->mlp_blob = blob;
    h->mlp_w1 = w1;
    h->mlp_w2 = w2;
    h->mlp_w3 = w3;
    h->guess = guess;
  }
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
  if (capacity > h->hcap) {  // grow: both buffers or neither; the old ones stay on failure
    float* nx = try_dalloc<float>(h, (size_t)capacity * MLP_IN);
    float* nt = nx ? try_dalloc<float>(h, (size_t)capacity * MLP_OUT) : nullptr;
    if (!nt) {
      dfree(h, nx);
      return reject(h, KC_ERR_OOM, h->err);
    }
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graph(h);
    dfree(h, h->hx);
    dfree(h, h->ht);
    h->hx = nx;
    h->ht = nt;
  }
  h->hcap = capacity;
  drop_graph(h);
  return cuda_check(h, cudaMemsetAsync(h->imp_ctr + 1, 0, 8, h->stream), "harvest reset");
}
// Which solves the harvest records (no reference counterpart): 0 every cell
// whose solve converged on the first rung, 1 only those among them whose
// pre-solve state fails the Newton core's first residual test (the cells a
// start from the pre-solve state would have to iterate).
int kc_set_harvest_filter(kc_handle* h, int32_t mode) {
  if (!h) return KC_ERR_INVALID_CONFIG;
  if (mode != 0 && mode != 1) return reject(h, KC_ERR_INVALID_CONFIG, "unknown harvest filter");
  h->harvest_filter = mode;
  drop_graph(h);
  return KC_OK;
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

#include "kc_abi_batch.inc"
#include "kc_abi_mlp.inc"
#include "kc_abi_fp64_peak.inc"
#include "kc_abi_autotune.inc"
#include "kc_abi_kdmp.inc"
