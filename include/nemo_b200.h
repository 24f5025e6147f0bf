/*
 * nemo_b200.h -- C ABI of the B200 (sm_100a) NEMOLite2D time-stepper.
 *
 * Two layers:
 *
 *  1. The handle API (nemo_*).  Every call returns an int status (NEMO_OK = 0)
 *     and never throws.  A context owns all device memory of one model
 *     instance and one CUDA stream; there is no global state.
 *
 *  2. Drop-in symbols with the exact names and signatures of the reference's
 *     CUDA library (cuda/cuda_nemolite2d.cu:234-270), bound from Fortran by
 *     cuda/nemolite2d.f90:62-127 (explicit bind(C) interfaces) and :138,
 *     :174, :486-489 (implicit interfaces with gfortran's trailing
 *     underscore).  They drive one process-wide default context.
 *
 * Field layout at the ABI edge is the reference's: Fortran column-major
 * arrays with the reference's bounds (ji fastest).
 *   T fields  (1:jpi, 1:jpj)   sshn, ssha, ht, xt, yt
 *   U fields  (0:jpi, 1:jpj)   un, ua, sshn_u, hu
 *   V fields  (1:jpi, 0:jpj)   vn, va, sshn_v, hv
 * (original/nemolite2d.f90:290-306).  Device storage is pitched and padded;
 * conversion happens in the copy routines below.
 */
#ifndef NEMO_B200_H
#define NEMO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum {
  NEMO_OK = 0,
  NEMO_ERR_INVALID = 1,     /* bad argument (size, field id, null pointer) */
  NEMO_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  NEMO_ERR_ALLOC = 3,       /* device or pinned allocation failed */
  NEMO_ERR_STATE = 4,       /* call out of order (e.g. no context) */
  NEMO_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  NEMO_ERR_UNSUPPORTED = 6  /* feature not available in this build/device */
};

/* ---- field identifiers ---------------------------------------------------- */
enum {
  NEMO_SSHN = 0, NEMO_UN = 1, NEMO_VN = 2,
  NEMO_SSHA = 3, NEMO_UA = 4, NEMO_VA = 5,
  NEMO_SSHN_U = 6, NEMO_SSHN_V = 7,
  NEMO_HT = 8, NEMO_HU = 9, NEMO_HV = 10,
  NEMO_XT = 11, NEMO_YT = 12,
  NEMO_NFIELDS = 13
};

/* Model parameters.  The first block is the reference's &namctl
 * (original/nemolite2d.f90:100-118; jpi/jpj are the namelist's jpiglo-2,
 * :133-137) and the argument list of cuda_setup_model_params_
 * (cuda/cuda_nemolite2d.cu:236-246).  The second block extends the
 * reference's hard-coded physics; nemo_default_params() sets values that
 * reproduce the reference exactly (amp_tide 0.2, phase 0, latitude 50,
 * uniform depth). */
typedef struct nemo_params {
  int jpi, jpj;
  double dx, dy, dep_const;
  int nit000, nitend, irecord;
  double rdt, cbfr, visc;
  /* extensions */
  double amp_tide;      /* original/nemolite2d.f90:629 hard-codes 0.2 */
  double tide_phase;    /* radians added to omega_tide*rtime */
  double lat;           /* gphiu/gphiv, :220-221 hard-code 50 */
  int nbump;            /* 0: uniform dep_const; >0: seeded Gaussian bumps */
  uint64_t seed;
  double bump_amp, bump_wmin, bump_wmax, hmin, hmax;
  /* execution */
  void* stream;         /* cudaStream_t to run on; NULL: the context makes one */
  int device;           /* CUDA device ordinal; -1: current device */
} nemo_params;

typedef struct nemo_ctx nemo_ctx;

/* Defaults of original/nemolite2d.f90:107-118 plus the extension defaults. */
int nemo_default_params(nemo_params* p);

/* grid + allocation + initialisation (original/nemolite2d.f90:145-371);
 * replaces cuda_setup_model_params_ + cuda_initialise_grid_
 * (cuda/cuda_nemolite2d.cu:418-446, :282-416).  jpi, jpj >= 2. */
int nemo_create(const nemo_params* p, nemo_ctx** out);
/* Frees everything the context owns; replaces cuda_finalise_ (:595-645),
 * without its cudaDeviceReset. */
int nemo_destroy(nemo_ctx* ctx);

/* ---- per-routine boundary (original/nemolite2d.f90:375-386) ---------------
 * Same semantics and order as the reference's routines; asynchronous on the
 * context's stream. */
int nemo_continuity(nemo_ctx* ctx);                /* :390-410; cu:448-476 */
int nemo_momentum(nemo_ctx* ctx);                  /* :414-613; cu:478-482 */
int nemo_momentum_u(nemo_ctx* ctx);                /* :430-517 */
int nemo_momentum_v(nemo_ctx* ctx);                /* :519-609 */
int nemo_bc(nemo_ctx* ctx, double rtime);          /* :617-700; cu:484-531 */
int nemo_bc_ssh(nemo_ctx* ctx, double rtime);      /* :626-645 */
int nemo_bc_solid_u(nemo_ctx* ctx);                /* :647-652 */
int nemo_bc_solid_v(nemo_ctx* ctx);                /* :655-660 */
int nemo_bc_flather_u(nemo_ctx* ctx);              /* :668-680 */
int nemo_bc_flather_v(nemo_ctx* ctx);              /* :683-695 */
int nemo_next(nemo_ctx* ctx);                      /* :704-769; cu:533-563 */
/* step (:375-386) without output: rtime = istp*rdt, then the four routines. */
int nemo_step(nemo_ctx* ctx, int istp);

/* ---- fused path -----------------------------------------------------------
 * Advances n steps istp0 .. istp0+n-1 with one fused launch per step
 * (continuity + momentum + bc + next in a single pass over HBM).  Results
 * equal nemo_step() called n times. */
int nemo_step_n(nemo_ctx* ctx, int istp0, int n);

/* Checksums SUM(ABS(f(1:jpi,1:jpj))) (shared/.../field_mod.f90:935-956,
 * original/nemolite2d.f90:82-85) of sshn, un (=ua after next) and vn (=va),
 * in out[0..2], computed on the device with a fixed reduction order. */
int nemo_checksums(nemo_ctx* ctx, double out[3]);
int nemo_checksum(nemo_ctx* ctx, int field, double* out);

/* Copies one field's Fortran-bounded region to/from host memory (column
 * major, leading dimension ld >= the field's x extent).  Replaces
 * cuda_retrieve_results_ / cuda_retrieve_grid_constants_ (cu:565-593).
 * These synchronise the context's stream. */
int nemo_retrieve(nemo_ctx* ctx, int field, double* host, long ld);
/* Output record of the current state for the model's go2d files
 * (original/nemolite2d.f90:773-799, which writes sshn and the cell-centred
 * velocities every irecord steps): a kernel stages sshn,
 * 0.5*(un(ji-1,jj)+un(ji,jj)) and 0.5*(vn(ji,jj-1)+vn(ji,jj)) at every T-cell
 * on the device, and one copy on a side stream moves them to `host`
 * ([3][jpj][jpi] FP64; pinned memory lets the copy overlap).  Returns at
 * once: later steps wait only for the staging kernel, so the stepper keeps
 * running while the record travels.  nemo_record_wait blocks until the last
 * record has landed in host memory.  Not a counterpart of a reference
 * routine: the reference copies whole fields back at every record. */
int nemo_record(nemo_ctx* ctx, double* host);
int nemo_record_wait(nemo_ctx* ctx);
/* Page-locked host memory for records and retrievals (callers that do not link
 * the CUDA runtime, e.g. Fortran or the C++ driver). */
int nemo_host_alloc(size_t bytes, void** ptr);
int nemo_host_free(void* ptr);
/* Overwrites sshn, un, vn (dense, Fortran extents) and re-derives
 * sshn_u/sshn_v with the post-`next` interpolation (:736-764); the
 * open-boundary row sshn_v(:,0), which the reference never updates after
 * initialisation, keeps its value.  The result is the state as after a
 * complete step: ssha, ua, va equal the new sshn, un, vn, as `next`
 * (:712-732) leaves them, so points that no routine of a step writes (a u
 * point between two open cells of a general grid) carry the given value. */
int nemo_set_state(nemo_ctx* ctx, const double* sshn, const double* un,
                   const double* vn);

/* A general grid in place of `grid`'s uniform one (original/nemolite2d.f90
 * :145-281): every array covers (0:jpi+1, 0:jpj+1), column-major (ji
 * fastest, leading dimension jpi+2), as the reference allocates its grid
 * arrays.  pt: 1 water, 0 land, -1 open water outside the domain (any cell of
 * the border ring may be open, so the Flather conditions on u and v can both
 * act, :669-695); e1t..e2v: scale factors (m); gphiu, gphiv: latitudes of
 * the u and v points (degrees); ht, hu, hv: depths, NULL keeps the
 * context's.  The reference fills each metric only over its own point set
 * and leaves the rest zero, which callers reproduce by passing zeros there.
 * Cell areas are formed over the ranges :263-279 fills, the Coriolis
 * parameter per point as the momentum loops form it, and sshn_u/sshn_v are
 * re-initialised from the current sshn (:337-353).  A context with a general
 * grid runs every step through the per-routine kernels (nemo_step_n
 * included; nemo_autotune answers NEMO_ERR_STATE): the fused kernel holds the
 * uniform grid's constants and analytic mask.  No counterpart in the
 * reference's CUDA library, whose grid is fixed. */
typedef struct nemo_grid {
  const int* pt;
  const double *e1t, *e2t, *e1u, *e2u, *e1v, *e2v;
  const double *gphiu, *gphiv;
  const double *ht, *hu, *hv;
} nemo_grid;
int nemo_set_grid(nemo_ctx* ctx, const nemo_grid* grid);

int nemo_sync(nemo_ctx* ctx);
int nemo_get_dims(nemo_ctx* ctx, int* jpi, int* jpj);
/* Device address and pitch (in doubles) of a field's storage; element
 * (ji,jj) lives at ptr[(jj+1)*pitch + (ji+2)].  For device-side consumers. */
int nemo_device_field(nemo_ctx* ctx, int field, double** ptr, long* pitch);
/* Launch schedule of the fused kernel: warps per CTA (2, 4, 8; a warp covers
 * 30 columns), register budget as resident warps per SM and row staging
 * (occupancy), and rows marched per CTA (0: one wave, row blocks sized so
 * every CTA is resident at once).  occupancy: 116 or 120 (2- and 4-warp
 * CTAs) stage rows through shared memory with a budget of 16 or 20 warps
 * (the default, 2 warps, 116, 16 rows); 0 (compiler's choice), 16, 20, 24
 * prefetch the next row into registers (8-warp CTAs take 0, 16 or 24); -16,
 * -20, -24 for 2-warp and -20 for 4-warp CTAs load each row one step ahead.
 * In the -fmad=false build every schedule gives bit-identical results.
 * After nemo_set_grid the context keeps a separate schedule for the general
 * grid's fused kernel: warps 2, occupancy 3 or 4 (rows staged through a
 * shared-memory ring of that many slots; 3 is the default) or 0 (each row
 * loaded where it is used), rows 1..65536 per CTA (default 32). */
typedef struct nemo_schedule {
  int warps;
  int occupancy;
  int rows;
} nemo_schedule;
int nemo_set_schedule(nemo_ctx* ctx, const nemo_schedule* s);
int nemo_get_schedule(nemo_ctx* ctx, nemo_schedule* s);
const char* nemo_status_string(int status);
/* 1 when this library was built with -fmad=false (bit-exact build). */
int nemo_build_is_strict(void);

/* ---- autotuning of the single-grid schedule ---------------------------------
 * No counterpart in the reference.  Times every compiled schedule variant
 * over `steps` fused steps (the model state is saved first and restored
 * afterwards, so results are unaffected), installs the fastest and returns
 * it.  With the environment variable NEMO_TUNE_CACHE naming a file, results
 * are stored there per (GPU, grid size) and nemo_create applies a stored
 * schedule. */
int nemo_autotune(nemo_ctx* ctx, int steps, nemo_schedule* best, double* best_ms_per_step);

/* ---- batched ensemble (no reference counterpart) ----------------------------
 * Many independent model instances of uneven size advanced together: one
 * persistent launch per step runs a work list of (member, column strip, row
 * block) items over every member, and the n launches of nemo_ens_step_n are
 * captured once in a CUDA graph and replayed.  Each member follows exactly
 * the single-grid arithmetic (same kernels, same results as a nemo_ctx with
 * the member's parameters). */
typedef struct nemo_member {
  int jpi, jpj;
  double amp_tide, tide_phase;
  double dep_const;
  int nbump;
  uint64_t seed;
  double bump_amp, bump_wmin, bump_wmax, hmin, hmax;
} nemo_member;

typedef struct nemo_ens nemo_ens;

typedef struct nemo_ens_schedule {
  int warps;      /* warps per CTA: 2 or 4 */
  int occupancy;  /* as nemo_schedule.occupancy: 116, 120 (2 warps), 116 (4
                     warps), 20, 24, -20, -24 (2 warps), 20, 24, -20 (4);
                     212, 216, 220 (2 warps) and 212, 216 (4 warps) stage rows
                     through shared memory with in-kernel reciprocal depths
                     at a budget of 12, 16, 20 resident warps per SM */
  int rows;       /* rows per work item */
  int order;      /* work-list order: 0 member by member, 1 largest member first,
                     2 dynamic: warps take the next item as they finish one,
                     items largest first (suits tall row blocks, e.g. 128) */
  int ctas;       /* persistent grid size; 0: every resident CTA slot */
} nemo_ens_schedule;

/* The batched configuration's member recipe: sides log-uniform in
 * [side_min, side_max], aspect ratio log-uniform in [0.5, 2], depth 100 m with
 * 8 Gaussian bumps clamped to [50, 150] m, tidal amplitude
 * amp_scale * U[0.5, 1.5] m and phase U[0, 2*pi), all drawn from seed. */
int nemo_ens_generate(uint64_t seed, int nmem, int side_min, int side_max, double amp_scale,
                      nemo_member* out);
/* common supplies dx, dy, rdt, cbfr, visc, lat, stream and device. */
int nemo_ens_create(const nemo_params* common, const nemo_member* members, int nmem,
                    nemo_ens** out);
int nemo_ens_destroy(nemo_ens* e);
int nemo_ens_step_n(nemo_ens* e, int istp0, int n);
/* out[3*m + k]: checksums of member m's sshn, un, vn (k = 0, 1, 2). */
int nemo_ens_checksums(nemo_ens* e, double* out);
int nemo_ens_retrieve(nemo_ens* e, int member, int field, double* host, long ld);
int nemo_ens_set_state(nemo_ens* e, int member, const double* sshn, const double* un,
                       const double* vn);
int nemo_ens_set_schedule(nemo_ens* e, const nemo_ens_schedule* s);
int nemo_ens_get_schedule(nemo_ens* e, nemo_ens_schedule* s);
/* Graph capture of nemo_ens_step_n on (1, default) or off (0). */
int nemo_ens_use_graph(nemo_ens* e, int on);
int nemo_ens_info(nemo_ens* e, int* nmem, long long* cells);
/* Times candidate schedules as nemo_autotune does, for the ensemble. */
int nemo_ens_autotune(nemo_ens* e, int steps, nemo_ens_schedule* best, double* best_ms_per_step);

/* ---- allocation-free checksums ----------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (all device memory owned by their own pool, or a loop that must not pay a
 * cudaMalloc's implicit device synchronisation): the checksums of
 * nemo_checksums, in the same fixed reduction order, from plain device
 * pointers, allocating nothing.  fields[k] points at element (1,1) of field k
 * (column major, leading dimension ld doubles); out is a device array of
 * nfields doubles; stream is a cudaStream_t (NULL: default stream).
 * Limits: nfields <= 4, ny <= NEMO_NOALLOC_MAX_ROWS (larger ny returns
 * NEMO_ERR_INVALID with a message on stderr).  Scratch is a fixed 512 KiB
 * device array inside the library, held on every GPU that loads it until the
 * process exits, and shared by all calls: calls that overlap on the GPU (for
 * instance on two streams at once) race on it.  The first call on each
 * device looks up the array's device address with that device current; make
 * that first call before any stream capture. */
#define NEMO_NOALLOC_MAX_ROWS 16384
int nemo_checksums_noalloc(const double* const* fields, int nfields, int nx, int ny,
                           long ld, double* out, void* stream);

/* ---- BF16 convolutional surrogate and hybrid controller ----------------------
 * No counterpart in the reference.  A residual CNN (nblocks blocks of two 3x3
 * convolutions, 64 channels, plus input and output convolutions) maps the
 * state of a grid at step s to its state at s + 10.  A snapshot is FP32
 * [n][height][width][4], one entry per T-cell (ji, jj) -> (x = ji-1,
 * y = jj-1): ssh(ji,jj), u(ji-1,jj) (west face), v(ji,jj-1) (south face),
 * ht(ji,jj).  The network's NHWC tensors hold one pixel per P x P patch of
 * T-cells (the configuration's patch).  Device pointers are the caller's;
 * every call is ordered on the configured stream. */
typedef struct nemo_sur nemo_sur;

typedef struct nemo_sur_config {
  int nblocks;          /* residual blocks (8) */
  int batch;            /* images per call (64) */
  int height, width;    /* grid (256 x 256) */
  int train;            /* 1: keep activations, gradients and AdamW moments */
  uint64_t seed;        /* weight initialisation */
  void* stream;         /* cudaStream_t; NULL: the surrogate creates one */
  int device;           /* -1: current device */
  int patch;            /* P = 1, 2 or 4: the network runs on P x P patches of
                           T-cells (height, width multiples of P; width / P a
                           multiple of 128); 0 means 1 */
} nemo_sur_config;

typedef struct nemo_adamw {
  float lr, beta1, beta2, eps, weight_decay;
} nemo_adamw;

int nemo_sur_default_config(nemo_sur_config* c);
int nemo_sur_create(const nemo_sur_config* c, nemo_sur** out);
int nemo_sur_destroy(nemo_sur* s);
/* Parameter count (FP32: all layers' weights [9][64 out][64 in], then all
 * biases [64]) and convolution FLOPs of one forward pass per T-cell (per
 * network pixel / P^2). */
int nemo_sur_info(nemo_sur* s, long long* nparams, long long* flops_per_pixel);
int nemo_sur_get_params(nemo_sur* s, float* host);
int nemo_sur_set_params(nemo_sur* s, const float* host);
int nemo_sur_get_grads(nemo_sur* s, float* host);
/* norm[11]: input scale[4], input shift[4] (ssh, u, v, depth; the tide channel
 * uses the ssh pair), output scale[3] (network output = delta * scale). */
int nemo_sur_set_norm(nemo_sur* s, const float* norm);
int nemo_sur_get_norm(nemo_sur* s, float* norm);
/* snap (device, [n][h][w][4] FP32 per T-cell: ssh, u west face, v south face,
 * depth); out (device, FP32): normalised deltas, [n][h][w][4] (channels
 * ssh, u, v, 0) for patch 1, else [n][h/P][w/P][3 P^2] with channel
 * f P^2 + P sy + sx = field f of T-cell (P X + sx, P Y + sy); tide[n] (device,
 * FP32): boundary-row SSH at the target time. */
int nemo_sur_predict(nemo_sur* s, const float* snap, const float* tide, int n, float* out);
/* Forward + mean-squared-error loss against snap1 + backward; gradients are
 * recomputed from zero.  loss: host double. */
int nemo_sur_loss_grad(nemo_sur* s, const float* snap0, const float* snap1, const float* tide,
                       int n, double* loss);
int nemo_sur_adamw(nemo_sur* s, const nemo_adamw* hp);
int nemo_sur_train_step(nemo_sur* s, const float* snap0, const float* snap1, const float* tide,
                        int n, const nemo_adamw* hp, double* loss);
/* Snapshot of every ensemble member (all must be height x width). */
int nemo_sur_pack_ens(nemo_sur* s, nemo_ens* e, float* snap);
/* One surrogate call: every member advances from its current state (after
 * step istp_end - k, k the step count the network was trained to advance,
 * 10 in the bundled recipe) to step istp_end; the boundary row takes the
 * exact tidal SSH, the walls keep zero normal velocity. */
int nemo_sur_advance_ens(nemo_sur* s, nemo_ens* e, int istp_end);
/* out[3*m + f]: relative L2 difference of member m's ssh, u, v (f) in a
 * against ref. */
int nemo_ens_compare(nemo_ens* a, nemo_ens* ref, double* out);

typedef struct nemo_hyb_config {
  int k;          /* steps per surrogate call: the step count the network
                     was trained to advance (10) */
  int anchor;     /* FP64 re-anchor interval (100) */
  double tol;     /* fallback threshold on relative SSH L2 error (0.01) */
  int per_member; /* 1: each member falls back on its own (anchor - k even);
                     0: any failing member sends the whole ensemble back (1) */
  double quarantine; /* shadow error beyond which a member stays on the FP64
                        solver for the rest of the run; 0: never (0.05) */
  int rewind;        /* 1: a quarantined member restarts from its FP64 state
                        at the start of the latest of the two previous
                        windows the surrogate advanced it in, the solver
                        re-running from there; after the last window a
                        member left non-finite or with |ssh| above 10 times
                        its tidal amplitude goes back to the start of the
                        latest of the last three windows the surrogate
                        advanced it in (keeps the states of the last three
                        window starts: 3 x 3 fields per member) (1) */
  int correct;       /* 1: every surrogate call of an accepted window also adds
                        the difference between the window's shadow state and
                        the surrogate's prediction of it, per cell (4 floats
                        per cell and member of device memory) (0) */
} nemo_hyb_config;

typedef struct nemo_hyb_stats {
  /* step counts are work done, windows a rewind discarded included */
  long long sur_calls;     /* surrogate calls (each advances its members k steps) */
  long long sur_steps;     /* member-steps advanced by the surrogate */
  long long solver_steps;  /* member-steps advanced by the FP64 solver */
  long long fallbacks;     /* member-windows that fell back to the solver */
  long long windows;       /* member-windows */
  double max_shadow_err, last_shadow_err;  /* worst member's shadow error */
  double seconds;
  long long launches;      /* kernels launched (solver steps and surrogate work) */
  long long quarantined;   /* members kept on the solver after a large shadow error */
  long long rewound;       /* quarantined members restarted from their previous anchor */
} nemo_hyb_stats;

int nemo_hyb_default_config(nemo_hyb_config* c);
/* Advances e by nsteps (a multiple of anchor) from the state after istp0.
 * Each anchor window: the surrogate predicts the first k steps while the
 * FP64 solver runs them (re-anchoring the state); each member whose relative
 * SSH L2 error of that prediction exceeds tol is advanced through the rest of
 * the window by the solver, the others by the surrogate, k steps per call. */
int nemo_hyb_run(nemo_sur* s, nemo_ens* e, const nemo_hyb_config* c, int istp0, int nsteps,
                 nemo_hyb_stats* stats);

/* Single convolution kernels on caller-owned device buffers.  x, out,
 * residual, mask, dz: BF16 NHWC, 64 channels; w: BF16 [9][64 out][64 in];
 * bias, dw ([9][64][64]), db ([64]): FP32; out32: FP32 [n][h][w][4] (first
 * four channels).  err: device int set non-zero if a device wait gave up.
 * fwd: out = epilogue(conv(x, w)) with v = acc + bias, += residual,
 * *= (mask > 0), relu.  wgrad: dw += x (*) dz, db += sum dz (accumulating). */
int nemo_conv3x3_fwd(const void* x, const void* w, const float* bias, const void* residual,
                     const void* mask, int relu, void* out, float* out32, int n, int h, int w_,
                     int* err, void* stream);
int nemo_conv3x3_wgrad(const void* x, const void* dz, float* dw, float* db, int n, int h, int w_,
                       int ctas, int* err, void* stream);
/* Process-wide forward kernel: 4 (default, with rows = 32) marches column
 * strips of `rows` output rows with each input row loaded once and multiplied
 * once per horizontal tap into all three output rows it feeds (N = 192 MMAs),
 * and each epilogue warp writes its 32 pixels of an output row with one TMA
 * store from shared memory; 2 is the same with per-thread stores; 3 is 2 with
 * two CTAs per SM (2 input-row slots, 256 TMEM columns each); 1 marches
 * the same strips with one N = 64 MMA per tap and output row; 0 loads one TMA
 * window per tap.  Returns the previous variant; values out of range change
 * nothing. */
int nemo_conv3x3_fwd_variant(int variant, int rows);
/* Process-wide weight-gradient kernel: 2 gives each CTA all nine
 * taps and the bias over a range of column-strip rows (one x window per row
 * read at three shifts, each dz row loaded once into a ring) and adds the
 * CTAs' partial sums in a fixed order afterwards, so results are
 * bit-identical from call to call; it keeps one scratch array per device for
 * nemo_conv3x3_wgrad (calls that overlap on the GPU race on it; a surrogate
 * has its own).  3 (default) is the same with 128-pixel column chunks instead
 * of 64 where the width is a multiple of 128 (else 2).  1 multiplies the x windows of two horizontal taps with the
 * dz windows of three rows (six taps per N = 192 MMA); 0 pairs taps with
 * N = 64 MMAs; both add partial results with atomics.  Returns the previous
 * variant; values out of range change nothing. */
int nemo_conv3x3_wgrad_variant(int variant);

/* ---- allocation-failure injection (tests of the error paths) ---------------
 * No counterpart in the reference, which stops the program when an ALLOCATE
 * fails (original/nemolite2d.f90:308).  Every device and page-locked
 * allocation of this library counts down from n: the n-th one from this call
 * on reports failure without allocating (n = 1: the next one), after which
 * the countdown is off again; n = 0 turns it off.  Returns the countdown's
 * previous value (so nemo_debug_fail_alloc(0) after a call tells whether the
 * failure fired: 0 yes, > 0 not reached), or -1 for n < 0.  Process-wide;
 * meant for tests, which check that every create call then returns
 * NEMO_ERR_ALLOC, sets no handle and leaves no device memory behind. */
int nemo_debug_fail_alloc(int n);

/* Test of the convolution kernels' failure path (no counterpart in the
 * reference).  The default forward kernel's main waits (operand rows, the
 * accumulator hand-over) give up after wait_ns nanoseconds of wall time
 * (0: the default, 2 s); the drains before exit keep 2 s.  The next
 * skip_launches forward launches leave out CTA 0's first input-row load, so
 * that the waits for that row run out: the kernel records an error code,
 * lets its copies and MMAs finish, frees its tensor memory and returns, and
 * the surrogate call reports NEMO_ERR_TIMEOUT.  Nothing faults and the
 * context stays usable.  Process-wide. */
int nemo_debug_conv_wait(unsigned long long wait_ns, int skip_launches);

/* ---- drop-in symbols (cuda/cuda_nemolite2d.cu:234-270) --------------------
 * One default context.  Errors are printed to stderr and kept in a sticky
 * status readable with nemo_compat_last_status() (the reference threw a C++
 * exception through the Fortran frames instead, cuda_utils.cuh:14-24). */
void cuda_setup_model_params_(int jpi, int jpj, double dx, double dy,
                              double dep_const, int nit000, int nitend,
                              int irecord, double rdt, double cbfr,
                              double visc);
void cuda_initialise_grid_(void);
void cuda_continuity_(void);
void cuda_momentum_(void);
void cuda_boundary_conditions_(double rtime);
void cuda_next_(void);
void cuda_retrieve_grid_constants_(double* out_xt, double* out_yt,
                                   double* out_ht, int jpi, int jpj);
void cuda_retrieve_results_(double* out_sshn, double* out_un, double* out_vn,
                            double* out_ua, double* out_va, int jpi, int jpj);
void cuda_finalise_(void);
int nemo_compat_last_status(void);
nemo_ctx* nemo_compat_context(void);

#ifdef __cplusplus
}
#endif
#endif
