/* koralcuda.h — the C ABI of libkoralcuda, the sm_100a GR-RMHD + M1 step engine.
 *
 * The reference (koral-zig) has no FFI: its step path sits behind the Zig
 * generic `Sim(cfg)` (koral/sim.zig:93). Each entry point below replaces one
 * method or field of that type, cited as file:line in koral-zig; a Zig host
 * binds them with `extern fn`. All structs are POD,
 * all arrays are caller-owned host memory copied at the call, and no call
 * aborts: every failure is an int status plus kc_last_error().
 *
 * Host array layout is the reference's Field layout (koral/field.zig:1-10):
 * AoS, variable fastest, signed cell indices including ghosts,
 *   offset = ((jz*SY + jy)*SX + jx)*NV + iv,  jx = ix + ngx, ...
 * with NV = 13 (RHO UU VX VY VZ ENTR B1 B2 B3 EE FX FY FZ) and ghosts
 * collapsed on size-1 dimensions (koral/grid.zig:17). Flags are six int32 per
 * cell (koral/sim/storage.zig:11): entropy, entropy2, entropy3, hd_fixup,
 * rad_fixup, radimp_fixup.
 */
#ifndef KORALCUDA_H
#define KORALCUDA_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KC_ABI_VERSION 1
#define KC_NV 13
#define KC_NFLAGS 6

/* status codes (the reference's relele.Error set, koral/relele.zig:51, plus
 * Sim.init's InvalidConfig, koral/sim.zig:319, and the device-side ones) */
enum {
  KC_OK = 0,
  KC_ERR_INVALID_CONFIG = 1,
  KC_ERR_OOM = 2,
  KC_ERR_VELOCITY_CONVERSION = 3,
  KC_ERR_SPACELIKE = 4,
  KC_ERR_NAN_IN_FLUX = 5,
  KC_ERR_CUDA = 6,
  KC_ERR_TIMEOUT = 7,
  KC_ERR_NO_DEVICE = 8,
  KC_ERR_TOO_MANY_CELLS = 9, /* more cells than kc_implicit_batch_noalloc stages */
  /* dump.zig:41 ReadError of the KDMP reader */
  KC_ERR_KDMP_BAD_MAGIC = 10,
  KC_ERR_KDMP_BAD_VERSION = 11,
  KC_ERR_KDMP_DIM_MISMATCH = 12,
  KC_ERR_KDMP_TRUNCATED = 13,
  KC_ERR_IO = 14 /* a KDMP file could not be opened, read or written */
};

enum { KC_BC_PERIODIC = 0, KC_BC_COPY = 1, KC_BC_PUFFY = 2 };
enum { KC_PLAIN_FP64 = 0, KC_MIXED = 1 };
/* The FP32 pieces of the mixed form, which kc_set_precision also takes one by
 * one or combined (no reference counterpart): the PPM reconstruction on
 * stencil deviations, the LAXF dissipation product, the flux-CT corner
 * averages, and the one-sided face fluxes rounded to FP32 (their arithmetic
 * stays FP64: the rounding alone bounds what FP32 flux arithmetic would do).
 * KC_MIXED is KC_FP32_LAXF | KC_FP32_CT: the pieces that keep the integrated
 * accretion rate and luminosity within 1e-4 of plain FP64 after 1000 steps of
 * the 192x180x64 wedge (the FP32 reconstruction alone moves them by 9e-3). */
enum { KC_FP32_PPM = 2, KC_FP32_LAXF = 4, KC_FP32_CT = 8, KC_FP32_FLUX = 16 };
enum { KC_GUESS_PLAIN = 0, KC_GUESS_MLP = 1 };
/* implicit pass forms (no reference counterpart; all bit-identical to the
 * reference's per-cell solveImplicitLab loop, koral/sim.zig:1715):
 * PER_CELL one thread per cell; COMPACTING a persistent lane-refilling state
 * machine; SPLIT an opening kernel that finishes every cell passing the Newton
 * core's first residual test at its warm start and a ladder kernel over the
 * compacted rest; SORTED (the batch entry points only) the per-cell kernel over
 * the cells sorted by start fluid, optical depth and temperature; RUNGS (the
 * batch entry points only) the sorted cells prepared once (warm start and
 * reference state), then one launch per rung of the ladder over the cells the
 * earlier rungs left unsolved, compacted between rungs; ITERS (the batch entry
 * points only) as RUNGS, with every rung run in launches of at most 8 Newton
 * iterations per cell, the cells still iterating compacted between launches */
enum {
  KC_IMPLICIT_PER_CELL = 0,
  KC_IMPLICIT_COMPACTING = 1,
  KC_IMPLICIT_SPLIT = 2,
  KC_IMPLICIT_SORTED = 3,
  KC_IMPLICIT_RUNGS = 4,
  KC_IMPLICIT_ITERS = 5
};

/* Pass ids of the per-pass timers, the members of koral/sim/timers.zig:4
 * Pass that the device step has. KC_PASS_FLUXES covers the reference's
 * `sweep` and `fluxes` passes, which the engine fuses into one face kernel;
 * KC_PASS_STEP is the untimed remainder of a step, as there. */
enum {
  KC_PASS_STEP = 0,
  KC_PASS_RADVISC,
  KC_PASS_IMPLICIT,
  KC_PASS_U2P,
  KC_PASS_FIXUP,
  KC_PASS_BC,
  KC_PASS_CORRECT,
  KC_PASS_WAVESPEEDS,
  KC_PASS_FLUXES,
  KC_PASS_FLUXCT,
  KC_PASS_UPDATE,
  KC_PASS_DYNAMO,
  KC_PASS_STAGE,
  KC_PASS_ENTROPY,
  KC_NPASS
};

/* koral/grid.zig:22 (Grid.init): internal-coordinate extents */
typedef struct kc_grid {
  int32_t nx, ny, nz, ng;
  double minx, maxx, miny, maxy, minz, maxz;
} kc_grid;

/* Sim.Options (koral/sim.zig:130) as built by the PUFFY problem's
 * Physics.toOptions (koral/problems/puffy/puffy.zig:210). */
typedef struct kc_options {
  int32_t abi_version;
  /* metric (koral/metric/forms.zig:16) and units (koral/units.zig:37) */
  double bhspin, mksr0, mksh0, mass;
  double gam, tsteplim, minmod_theta;
  /* FloorParams (koral/solve/invert.zig:60) */
  double rhofloor, uurhoratiomin, uurhoratiomax, b2rhoratiomax, b2uuratiomax, gammamaxhd;
  int32_t isentropic_b2rhofloors, b2uufloor;
  double horizon_x1;
  /* RadParams (koral/solve/invert_rad.zig:36) */
  double gammamaxrad, eradfloor, eerhoratiomin, eerhoratiomax, eeuuratiomin, eeuuratiomax;
  /* opacity channels and composition (koral/physics/opacities.zig:61, thermo.zig:33) */
  int32_t bremsstrahlung, synchrotron, kleinnishina, comptonization, synchrotron_bridge;
  int32_t scattering; /* Klein-Nishina kappa_es hook on/off (PR_KAPPAES) */
  double hfrac, hefrac, mu_gas, mu_i, mu_e;
  /* ImplicitParams (koral/solve/implicit.zig:83) */
  double radimp_conv, radimp_entrconv, radimp_eps;
  int32_t radimp_maxiter;
  double radimp_convrel, radimp_convrelerr, radimp_convrelentr, radimp_convrelentrerr;
  double radimp_damping_factor, radimp_max_en_change_down, radimp_max_en_change_up, radimp_max_damping;
  double radimp_max_tgas_change, radimp_max_trad_change, radimp_threshold;
  int32_t radimp_start_with_bisect, radimp_scale_jacobian, radimp_allow_rad_ceiling, radimp_allow_entr_in_4dprim;
  int32_t radimp_opdamp_maxlevels;
  double radimp_opdamp_factor;
  int32_t radimp_lag_opac;
  /* fixups, polar axis, radiative viscosity, dynamo (koral/sim.zig:150-180) */
  int32_t do_fixups, do_u2prad_fixups, do_radimp_fixups;
  int32_t correct_polaraxis, nccorrectpolar;
  int32_t radviscosity;
  double alpharadvisc, maxradviscvel;
  int32_t dynamo;
  double alphadynamo, thetaangle, alphabeta, betasaturated, expectedhr;
  int32_t alphaflipssign, dampbeta, calchronthego;
  int32_t reduceorderatbh, reduceorderafterfixup, dampradwavespeednearaxis;
  int32_t bc_x, bc_y, bc_z;
  /* engine forms (no reference counterpart) */
  int32_t precision;     /* KC_PLAIN_FP64, KC_MIXED, or a set of KC_FP32_* pieces */
  int32_t implicit_mode; /* KC_IMPLICIT_PER_CELL | KC_IMPLICIT_COMPACTING | KC_IMPLICIT_SPLIT */
  int32_t device;        /* CUDA device ordinal */
} kc_options;

/* Sim counters and step scalars (koral/sim.zig:237-293, invert.zig:44) */
typedef struct kc_counters {
  double t, dt, own_dt, tstepdenmax, tstepdenmin;
  int64_t nstep;
  int64_t n_radimp_failures, n_radimp_fail_step, n_radimp_iters, n_radimp_solves;
  int64_t n_guard_recoveries;
} kc_counters;

typedef struct kc_step_info {
  double dt;
  int64_t nan_cell; /* first flat cell index whose face flux was non-finite, or -1 */
} kc_step_info;

typedef struct kc_handle kc_handle;

/* Fills the PUFFY option set (puffy.zig:210 toOptions with Physics defaults,
 * puffy.zig:84). */
void kc_options_puffy(kc_options* opt);
/* The PUFFY grid (puffy.zig:179 makeGridNz). */
void kc_grid_puffy(int32_t nx, int32_t ny, int32_t nz, kc_grid* grid);

/* Sim.init (koral/sim.zig:309): validates, builds the metric cache and
 * allocates the device state. */
int kc_create(const kc_grid* grid, const kc_options* opt, kc_handle** out);
/* Sim.deinit (koral/sim.zig:501) */
void kc_destroy(kc_handle* h);
const char* kc_last_error(const kc_handle* h);

/* Sim.p / Sim.u / Sim.flags field access (koral/sim.zig:224-262) */
int kc_upload_prims(kc_handle* h, const double* p_aos);
int kc_upload_cons(kc_handle* h, const double* u_aos);
int kc_upload_flags(kc_handle* h, const int32_t* flags);
int kc_download_prims(kc_handle* h, double* p_aos);
int kc_download_cons(kc_handle* h, double* u_aos);
int kc_download_flags(kc_handle* h, int32_t* flags);
/* restores t, dt, tstepdenmax/min and the counters (restart / replay) */
int kc_set_counters(kc_handle* h, const kc_counters* c);
int kc_get_counters(kc_handle* h, kc_counters* c);

/* One row of the diagnostics time series (koral/io/dump.zig:414 ScalarRow),
 * code units: mass (scalars.zig:78 totalMass), mdot through the horizon shell
 * (>0 for accretion, scalars.zig:106), radiative and total luminosity through
 * the shell at r_lum in BL (scalars.zig:136, type 1), density-weighted scale
 * height at r_scale (dynamo.zig:239), max pmag/ptot (scalars.zig:276), and the
 * counts of dump.zig:358 collectDiag plus the solver counters. */
typedef struct kc_scalar_row {
  double t, dt;
  int64_t nstep;
  double mass, mdot, radlum, totallum, scaleheight, max_pmag_ptot;
  int64_t n_hd_fixup, n_radimp_fail, n_nan, n_floorguard;
} kc_scalar_row;

/* PUFFY initial state: puffy.initAllWith (koral/problems/puffy/puffy.zig:873)
 * — limotorus, atmosphere, A_phi seed, set_bc, B from A, set_bc, beta
 * normalization — followed by Sim.initTimestepGuess, as
 * koral/problems/puffy/main.zig:304-305 does; t and the counters restart at 0.
 * perturb is the relative u_int noise amplitude of puffy.zig:750 (Physics
 * .perturb), perturb_rho the same for rho (no reference counterpart; 0 leaves
 * the reference's init unchanged); seed is XORed into the x1 word of the
 * per-cell hash (puffy.zig:696 perturbXi; 0 is the reference's field, rho uses
 * seed ^ 0x5DEECE66D). fac_out (may be NULL) receives the normalization
 * factor sqrt(maxbeta / max beta) that initAllWith returns. */
int kc_init_puffy(kc_handle* h, double perturb, double perturb_rho, uint64_t seed, double* fac_out);
/* dump.scalarRow (koral/io/dump.zig:383) on the current state; `dt` is only
 * recorded. PUFFY's driver uses r_lum = 5000, r_scale = 15
 * (koral/problems/puffy/main.zig:30). The sums are folded in the reference's
 * serial cell order, so the row is bit-identical to a serial evaluation. */
int kc_scalars(kc_handle* h, double dt, double r_lum, double r_scale, kc_scalar_row* out);
/* Sim.finishInit (koral/sim.zig:686): ghost fill from p, then the dt guess */
int kc_finish_init(kc_handle* h);
/* Sim.initTimestepGuess (koral/sim.zig:693) */
int kc_init_timestep_guess(kc_handle* h);
/* Sim.setBc / Sim.calcU2p (koral/sim.zig:735, :924) */
int kc_set_bc(kc_handle* h);
int kc_calc_u2p(kc_handle* h);
/* Sim.cflDt (koral/sim.zig:726) */
int kc_cfl_dt(kc_handle* h, double* dt);
/* Sim.step (koral/sim.zig:1792): forced_dt NaN means the CFL dt. */
int kc_step(kc_handle* h, double forced_dt, kc_step_info* info);
/* host buffers -> step(s) -> host buffers in one call */
int kc_step_n(kc_handle* h, int32_t nsteps, double forced_dt);

/* Sim.timers (koral/sim/timers.zig:41 PassTimers): per-pass self time of the
 * steps taken while timing is on, measured on the device with CUDA events at
 * every pass boundary of the handle's stream. kc_set_pass_timing resets the
 * totals; kc_get_pass_times fills KC_NPASS entries of milliseconds and of
 * pass calls (either pointer may be NULL). */
int kc_set_pass_timing(kc_handle* h, int32_t on);
int kc_get_pass_times(kc_handle* h, double* ms, int64_t* calls);
const char* kc_pass_name(int32_t pass);
/* The handle's CUDA stream (a cudaStream_t), on which every step kernel is
 * launched, and the number of kernels the step passes have launched since
 * kc_create (no reference counterpart: device plumbing for callers that time
 * or order work against the engine). */
int kc_get_stream(kc_handle* h, void** stream);
int kc_get_launch_count(kc_handle* h, int64_t* n);

/* Engine forms (no reference counterpart) */
int kc_set_precision(kc_handle* h, int32_t mode);
/* Selecting KC_IMPLICIT_SPLIT allocates that form's compact list; when that
 * fails the call returns KC_ERR_OOM and the form stays as it was. */
int kc_set_implicit_mode(kc_handle* h, int32_t mode);
/* Test hook (no reference counterpart): the n-th next optional allocation (of
 * the split form's list, the learned guess's buffers, the harvest records and
 * their counters) fails as if the device were full, so the call that makes it
 * returns KC_ERR_OOM with nothing half-allocated kept; 0 disarms. */
int kc_debug_fail_allocs(kc_handle* h, int32_t n);
/* The step as a CUDA graph: with on != 0 the whole step's launch sequence
 * (every pass of koral/sim.zig:1792 step, and the copy of its dt-derived
 * coefficients from a pinned table) is captured once and replayed each step;
 * results are bit-identical to the eager launches. The step after a change of
 * form (precision, implicit form, guess, harvest) runs eagerly, the next one is
 * captured. Pass timing (kc_set_pass_timing) runs the steps eagerly. */
int kc_set_graph(kc_handle* h, int32_t on);
/* The y and z face sweeps' form (no reference counterpart; every form gives the
 * same bits): 0 one thread per face reconstructing both of its neighbour cells
 * (the default), 1 blocks of 32 columns x 4 faces that reconstruct each cell
 * once into shared memory, 2 the same with the PPM stencil rows staged in
 * shared memory too. kc_autotune picks among them. */
int kc_set_face_tiles(kc_handle* h, int32_t mode);
/* Threads per block of the per-cell implicit kernel (no reference counterpart;
 * every size gives the same bits): one block fills an SM, so the size sets the
 * register budget: 256 (255 registers per thread, 8 warps), 384 (168, 12 warps;
 * the default) or 512 (128, 16 warps). Other sizes: KC_ERR_INVALID_CONFIG.
 * kc_autotune picks among them. */
int kc_set_implicit_threads(kc_handle* h, int32_t threads);

/* The autotuner's choice (no reference counterpart): implicit form
 * (KC_IMPLICIT_PER_CELL or KC_IMPLICIT_SPLIT), threads per block of the
 * per-cell implicit kernel (one block per SM: 256 threads with 255 registers
 * each, 384 with 168, 512 with 128), of the face-flux and of the u2p kernels,
 * the per-cell implicit kernel's thread -> cell order (1, the default: phi
 * fastest on 3D grids, so that a warp's cells share r and theta, theta fastest
 * on 2D grids; 0: x fastest) and whether the y and z face sweeps stage their
 * PPM stencils in shared-memory tiles, with the measured step time of the
 * choice and of the configuration on entry. */
typedef struct kc_tune_result {
  int32_t implicit_mode, tpb_implicit, tpb_flux, tpb_u2p;
  double ms_per_step, ms_per_step_entry;
  int32_t trials;
  int32_t implicit_phi_fastest;
  int32_t implicit_warps; /* warps per SM of the per-cell implicit kernel: tpb_implicit / 32 */
  int32_t face_tiles;          /* the y and z face sweeps' form (kc_set_face_tiles) */
} kc_tune_result;
/* Times whole steps on the handle's current state for each candidate, one
 * knob at a time, and keeps the fastest configuration set; the state and the
 * counters are restored afterwards, and all candidates are bit-identical.
 * `steps` timed steps per trial (after one untimed step, two with the graph
 * form). Not with the learned guess, the harvest or pass timing on. */
int kc_autotune(kc_handle* h, int32_t steps, kc_tune_result* out);

/* The learned initial guess of the implicit solve (no reference counterpart).
 * A 16 -> 64 -> 64 -> 4 ReLU network predicts, from a cell's pre-solve
 * primitives, the four Newton unknowns of the start fluid; the FP64 Newton
 * ladder then starts from that state instead of the bisection warm start of
 * koral/solve/implicit.zig:944, and the plain solve runs when the seeded ladder
 * fails. Weights are one FP32 blob of KC_MLP_NWEIGHTS floats: input mean[16],
 * input std[16], output mean[4], output std[4], W1[64][16], b1[64],
 * W2[64][64], b2[64], W3[4][64], b3[4] (row-major [out][in]). Inference runs
 * on the tensor cores with BF16 weights and activations and FP32
 * accumulation. Features (before standardisation): log10 rho, log10 u_int,
 * asinh(1e3 v^i), +1/-1 for a gas/radiation start, asinh(1e12 B^i),
 * log10 E_rad, asinh(1e3 F^i), log10 dt, log10 sqrt(-g), alpha. Targets:
 * asinh(ln(e_sol / e_0) / 1e-7) for the start fluid's energy density and
 * asinh((v_sol - v_0) / max(1e-6, |v_0|) / 1e-9) for its velocities (the
 * changes in the units of the Newton convergence test, compressed).
 * kc_set_guess(KC_GUESS_MLP) installs the weights for the handle's steps
 * (KC_GUESS_PLAIN returns to the reference path). The learned guess and the
 * harvest run the per-cell implicit form. */
enum { KC_MLP_IN = 16, KC_MLP_HIDDEN = 64, KC_MLP_OUT = 4, KC_MLP_NWEIGHTS = 5548 };
int kc_set_guess(kc_handle* h, int32_t mode, const float* weights, int64_t nweights);
/* Training pairs from the handle's own steps: from the next implicit pass on,
 * each cell whose solve converged on the first rung stores its features and
 * targets, up to `capacity` pairs (0 stops the harvest); kc_get_harvest copies
 * the pairs collected so far out and sets *n. */
int kc_harvest_implicit(kc_handle* h, int64_t capacity);
/* Which solves the harvest records: 0 (default) every cell whose solve
 * converged on the first rung; 1 only those whose pre-solve state fails the
 * Newton core's first residual test, i.e. the cells a start from the pre-solve
 * state (the reference's radimp_start_with_bisect = 0) would iterate. */
int kc_set_harvest_filter(kc_handle* h, int32_t mode);
int kc_get_harvest(kc_handle* h, float* features, float* targets, int64_t capacity, int64_t* n);
/* seeded ladders that failed and fell back to the plain solve, since the
 * guess was first installed */
int64_t kc_guess_fallbacks(kc_handle* h);
/* Trains the network on the GPU (FP32 forward/backward kernels with the
 * weights rounded to BF16 in the forward pass, Adam): normalisation from the
 * pairs (feature deviations floored at 0.01; standardised features clipped to
 * +-8, as the guess clips its inputs and outputs), He-uniform start from
 * `seed`, `steps` minibatches of `batch` pairs.
 * weights_out gets the blob; loss_curve (may be NULL) the mean squared error
 * of each step's minibatch in standardised units. Host arrays. */
int kc_mlp_train(const float* features, const float* targets, int64_t n, int32_t steps, int32_t batch, float lr,
                 uint64_t seed, float* weights_out, float* loss_curve);
/* The tensor-core forward pass on standardised features (n x 16) into
 * standardised outputs (n x 4); and the training kernels' loss (mean squared
 * error) and its gradient with respect to the blob (entries before W1 are
 * zero) over all n pairs. Host arrays. */
int kc_mlp_forward(const float* weights, int64_t n, const float* features_std, float* out_std);
int kc_mlp_grad(const float* weights, int64_t n, const float* features_std, const float* targets_std, float* grad,
                float* loss);

/* KDMP v2 checkpoints (koral/io/dump.zig): a 44-byte little-endian header
 * (magic "KDMP", version 2, nx ny nz nv as u32, t f64, nstep u64, out_idx u32;
 * dump.zig:29 DumpHeader, :38 header_size) followed by the domain primitives
 * p[nz][ny][nx][nv] as f64, iv fastest (dump.zig:100 serializePrimDump). */
#define KC_KDMP_HEADER_SIZE 44
#define KC_KDMP_VERSION 2
typedef struct kc_dump_header {
  uint32_t nx, ny, nz, nv;
  double t;
  uint64_t nstep;
  uint32_t out_idx;
} kc_dump_header;
/* writeDumpHeader (dump.zig:67) into out[KC_KDMP_HEADER_SIZE]; host only */
int kc_kdmp_write_header(const kc_dump_header* hd, uint8_t* out);
/* parseDumpHeader (dump.zig:86): magic, version and length checked; host only */
int kc_kdmp_parse_header(const uint8_t* bytes, int64_t len, kc_dump_header* hd);
/* primDumpSize (dump.zig:45) of the handle's grid */
int64_t kc_kdmp_size(kc_handle* h);
/* serializePrimDump (dump.zig:100) of the device state: the domain is gathered
 * into AoS order on the device and copied out once; t and nstep from the
 * handle. `capacity` must be at least kc_kdmp_size. */
int kc_kdmp_write(kc_handle* h, uint32_t out_idx, uint8_t* out, int64_t capacity, int64_t* written);
/* loadPrimDump (dump.zig:143): header checks (dims against the handle's grid),
 * then per domain cell p = the stored primitives and u = p2u(p) on the device,
 * as Sim.initCell (koral/sim.zig:672) does. As in the reference, the caller
 * adopts t / nstep from *hd (kc_set_counters) and runs kc_finish_init. */
int kc_kdmp_load(kc_handle* h, const uint8_t* bytes, int64_t len, kc_dump_header* hd);
/* writePrim / loadPrim (dump.zig:213, :270), serial: the same through a file */
int kc_kdmp_write_file(kc_handle* h, const char* path, uint32_t out_idx);
int kc_kdmp_load_file(kc_handle* h, const char* path, kc_dump_header* hd);

/* The FP64 pipe's peak on the current device, measured: independent DFMA
 * chains over every SM, best of five launches, in TFLOP/s (the denominator of
 * the FP64 roofline of the implicit solve and u2p; no reference counterpart). */
int kc_fp64_peak(double* tflops);

/* Batched per-cell entry points over n independent cells (the C4 implicit
 * microbench and the parity harnesses). geom23 is the reference's golden
 * record geometry (gg upper triangle, GG upper triangle, gdet, alpha,
 * gttpert; koral/testing/golden.zig:241). Arrays are host memory, cell-major.
 * solveImplicitLab (koral/solve/implicit.zig:927): pp is in/out, res is
 * {ok, rung, iters, whichprim, whicheq, whichframe} per cell. */
int kc_implicit_batch(const kc_options* opt, int64_t n, const double* geom23, const double* dt, double* pp,
                      int32_t* res, int32_t mode);
/* kc_implicit_batch on device arrays: geom23, dt, pp and res are device
 * pointers, the launch goes to `stream` (a cudaStream_t, NULL = default) and
 * the call returns without waiting (no counterpart in the reference: the
 * GPU-resident form of the same batch). */
int kc_implicit_batch_device(const kc_options* opt, int64_t n, const double* geom23, const double* dt, double* pp,
                             int32_t* res, int32_t mode, void* stream);
/* Seeded synthetic cells for the batched implicit-solve microbenchmark (no
 * reference counterpart; the distribution widens the reference's battery,
 * tools/bench_implicit.zig): MKS2 geometry at r log-uniform in [3, 50] and
 * theta uniform in [0.3, pi-0.3]; rho log-uniform in [1e-8, 1]; T_gas
 * log-uniform in [1e5, 1e9] K; |v| < 0.9c in a random direction; B with beta
 * log-uniform in [1, 1e3]; E_gas/E_rad log-uniform in [1e-4, 1e4]; radiation
 * frame Lorentz factor in [1, 2]; dt log-uniform in [1e-10, 1]. Host arrays. */
int kc_synth_implicit_cells(const kc_options* opt, int64_t n, uint64_t seed, double* geom23, double* dt, double* pp);
/* kc_implicit_batch without any allocation (no counterpart in the reference):
 * for callers that cannot allocate device memory, such as a host application
 * whose device memory is owned by another allocator (a framework's caching
 * allocator holding the device) or a fixed-budget process. The arrays are
 * staged through one fixed device array of KC_NOALLOC_MAX_CELLS cells (5 MiB),
 * held by every device that loads the library until exit; n above the maximum
 * returns KC_ERR_TOO_MANY_CELLS. Only mode KC_IMPLICIT_PER_CELL is accepted
 * (others return KC_ERR_INVALID_CONFIG: those forms need stream-ordered
 * scratch). The first call on a device looks up that array's address with the
 * device current. Every call is synchronous (blocking copies and a device
 * synchronize), so none may be made while a stream capture is active on the
 * device. Calls share the array: calls that overlap on one device race. */
#define KC_NOALLOC_MAX_CELLS 16384
int kc_implicit_batch_noalloc(const kc_options* opt, int64_t n, const double* geom23, const double* dt, double* pp,
                              int32_t* res, int32_t mode);
/* ct.fluxCt (koral/sim/ct.zig:38-177) on given face fluxes, without a handle,
 * on `device`: fb_x/fb_y/fb_z hold the B1, B2, B3 rows of the x/y/z face
 * fluxes of an nx x ny x nz domain with ng ghost layers, in the reference's
 * FaceStore layout (koral/sim/storage.zig:62: the face direction has one more
 * slice, ghosts included, offset = ((jz*FY + jy)*FX + jx)*3 + k with
 * FX = SX + (dir == x) etc.); the corner EMFs are formed and the B rows
 * rebuilt in place, as the step's flux-CT pass does. An inactive direction's
 * array may be NULL. */
int kc_flux_ct(int32_t device, int32_t nx, int32_t ny, int32_t nz, int32_t ng, double* fb_x, double* fb_y,
               double* fb_z);
/* u2p cascade of one cell as calcU2p applies it (koral/sim.zig:972-994):
 * u2pMhd + u2pRad + both floors. flags_out: {entropy_used, hd_fixup, rad_fixup} */
int kc_u2p_batch(const kc_options* opt, int64_t n, const double* geom23, const double* uu, double* pp,
                 int32_t* flags_out);

#ifdef __cplusplus
}
#endif
#endif
