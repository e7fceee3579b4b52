/*
 * mcs.h -- C ABI of libmcs.so, the B200 (sm_100a) time-domain regenerative-chatter
 * stability library.
 *
 * The library replaces the JavaScript hot path of the machining simulator:
 *   - chatterAt / timeDomainLimit          src/stabtd.js:14-32
 *   - the CuttingEngine force law, modal
 *     integration and chatter index they
 *     run per trial                         src/cutting.js:39-124,146-296,299-318
 *   - the stability Web Worker's sweep     src/stabworker.js:6-14
 *   - zero-order lobes / alimAt            src/sld.js:6-76
 *
 * All inputs and outputs are caller-owned host arrays of the plain structs below
 * (structure-of-records, no pointers inside).  Units follow the reference engine:
 * lengths in mm, modal stiffness in N/mm, frequencies in Hz, runout in mm.
 * Every entry point returns an mcs_status; on failure mcs_last_error() holds a
 * message for the calling thread.  There is no CPU fallback: without a CUDA device
 * the calls fail with MCS_ERR_CUDA.
 *
 * Thread safety: a context may be shared between threads; calls on one context are
 * serialised by a mutex inside it.
 */
#ifndef MCS_H_
#define MCS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCS_ABI_VERSION 2 /* 2: mcs_guide_opts gained mode, levels and skip_top;
                             mcs_guide_info reports rounds */
#define MCS_MAX_MODES 4 /* modes per axis (frf.js fitModes keeps at most 4) */
#define MCS_MAX_TEETH 8
#define MCS_BINS 180    /* angular bins of the engagement map, cutting.js:15 */

typedef enum {
  MCS_OK = 0,
  MCS_ERR_ARG = 1,         /* invalid argument (sizes, indices, NaN, out-of-range values) */
  MCS_ERR_CUDA = 2,        /* CUDA runtime error or no device */
  MCS_ERR_TIMEOUT = 3,     /* a bounded device wait gave up */
  MCS_ERR_DIVERGED = 4,    /* NaN/Inf in a simulated trial (per point) */
  MCS_ERR_CANCELLED = 5,   /* the job was cancelled before this point ran */
  MCS_ERR_NOMEM = 6,       /* allocation failed */
  MCS_ERR_UNSUPPORTED = 7, /* a case the kernels do not handle (e.g. > 64 slices) */
  MCS_ERR_STATE = 8        /* call out of order (e.g. results of a plan never run) */
} mcs_status;

typedef enum { MCS_TOOL_FLAT = 0, MCS_TOOL_BALL = 1 } mcs_tool_type;

/* Arithmetic of the per-step force law and modal integration.  The once-per-tooth
 * statistics, the chatter index and the bisection bracket are FP64 in both; the surface
 * ring is float in both (the reference's Float32Array).  MCS_FP64, the default, is the
 * reference's own arithmetic; MCS_FP32 runs about 1.6x faster, and its limits land within
 * 2 % of the FP64 reference about as often as the reference's own do when its feed is
 * changed by 1e-6 (near chaotic chatter the limits are ill-conditioned). */
typedef enum { MCS_FP32 = 0, MCS_FP64 = 1 } mcs_precision;

/* One mode of the tool tip: frf.js:1-11 {k [N/mm], fn [Hz], zeta}. */
typedef struct {
  double k;
  double fn;
  double zeta;
} mcs_mode;

/* Modal set of the tool tip, frf.js modeSet: ny == 0 means y takes the x modes. */
typedef struct {
  int32_t nx;
  int32_t ny;
  mcs_mode x[MCS_MAX_MODES];
  mcs_mode y[MCS_MAX_MODES];
} mcs_modal;

/* Tool as CuttingEngine.configure reads it (cutting.js:39-44). */
typedef struct {
  int32_t N;           /* flutes, 1..MCS_MAX_TEETH */
  int32_t type;        /* mcs_tool_type */
  double R;            /* radius [mm] */
  double helix_deg;    /* helix angle [deg] */
  double flute_len;    /* flute length [mm] */
  double runout;       /* radial runout e [mm] */
  double runout_phase; /* runout phase gamma [rad] */
} mcs_tool;

/* Cutting coefficients, materials.js:2-14 (Kac/Kae act only on Fz and are not needed). */
typedef struct {
  double Ktc, Krc; /* shearing [N/mm^2] */
  double Kte, Kre; /* edge [N/mm] */
  double mc;       /* size-effect exponent */
  double Ci;       /* process-damping coefficient [N/m] */
} mcs_material;

/* Everything of a cut except the speed and the modes. */
typedef struct {
  mcs_tool tool;
  mcs_material mat;
  double arc_st, arc_ex; /* engagement arc [rad], identify.js immersion() */
  double fz;             /* feed per tooth [mm] */
} mcs_setup;

/* One boundary point: a setup at a spindle speed with the modal set at that speed
 * (the Worker message carries one modal per point, stabworker.js:10 / main.js:496). */
typedef struct {
  uint32_t setup;
  uint32_t modal;
  double S; /* spindle speed [rpm] */
} mcs_point;

/* Options of timeDomainLimit/chatterAt (stabtd.js:14,24) plus explicit overrides. */
typedef struct {
  double a_min, a_max;     /* bisection range [mm] (reference 0.05, 20) */
  int32_t iters;           /* bisection iterations (reference 8) */
  int32_t revs;            /* revolutions per trial (reference 120) */
  int32_t nonlinear;       /* size effect + process damping (reference 1) */
  int32_t honor_runout;    /* 0: runout forced to 0 as chatterAt does (stabtd.js:16) */
  int32_t steps_per_tooth; /* 0: reference rule max(48, ceil(Ttooth*fTop*24)) */
  int32_t slices;          /* 0: reference rule dz = max(0.25, fluteLen/48) */
  double chatter_idx;      /* decision threshold (reference 0.45, stabtd.js:10) */
  int32_t precision;       /* mcs_precision of the force law and modal integration */
  int32_t max_buckets;     /* schedule: at most this many shared-memory size classes, each
                              its own persistent grid (1..MCS_MAX_BUCKETS; 0: 16), besides
                              one grid per block width of the multi-warp points (coop_warps);
                              results do not depend on it, only the time does (see
                              mcs_tune) */
  int32_t serial_trials;   /* 0: a bisection runs the trials of its next levels together in
                              lane groups of one warp when their slice counts allow
                              (speculatively; only the trials on the decision path count);
                              1: one trial at a time.  Results are identical either way. */
  int32_t coop_warps;      /* schedule: the heaviest points share their bisection among this
                              many warps of one block, each running one trial of the next
                              levels speculatively (2..8, narrowed to 4 or 3 where the rings
                              do not fit in shared memory; 1: off; 0: the library's rule,
                              see coop_points).  Plain solves only.  Results are identical
                              either way. */
  int32_t coop_points;     /* schedule: how many of the costliest points take that path
                              (0: one per SM).  With coop_warps and coop_points both 0 the
                              library's rule applies: 8 warps (or the widest that fits) for
                              each point whose serial bisection costs more than the batch's
                              share of one resident warp -- the points that would still run
                              once the device has done the rest -- up to two per SM; none
                              in a batch bound by its total work.  Points whose trials
                              share a warp in lane groups (all of them in at most half a
                              warp) keep that instead. */
  int32_t pad;
} mcs_opts;

#define MCS_MAX_BUCKETS 32

/* Result of timeDomainLimit for one point. */
typedef struct {
  double alim;          /* critical depth [mm] */
  double lo, hi;        /* bracket [stable, chatter]; hi = +inf when open */
  int32_t open;         /* 1 when stable at a_max (bracket[1] === Infinity) */
  int32_t status;       /* mcs_status of this point */
  int32_t trials;       /* trials run */
  int32_t steps_per_tooth;
  uint64_t evals;       /* reference-loop slice evaluations (steps * N * nz summed) */
  uint64_t engaged;     /* of which in cut (force evaluated) */
} mcs_result;

/* One chatterAt trial: a point at an axial depth. */
typedef struct {
  uint32_t point;
  uint32_t pad;
  double ap; /* [mm] */
} mcs_trial;

/* chatterIndex() of one trial (cutting.js:299-318) and the decision. */
typedef struct {
  double index;
  double once; /* sOnce [um] */
  double amp;  /* sAll [um] */
  int32_t chatter;
  int32_t status;
} mcs_trial_result;

/* Zero-order lobe query, the argument object of stabilityLobes (sld.js:23). */
typedef struct {
  int32_t N;
  int32_t lobes;
  double Ktc, Krc;
  double phi_st, phi_ex;
  double rpm_min, rpm_max;
  uint32_t modal; /* index into modals */
  uint32_t pad;
} mcs_lobe_query;

/* Launch and work figures of a plan, for measurement. */
typedef struct {
  int32_t blocks;        /* persistent CTAs launched */
  int32_t warps_per_sm;  /* resident warps per SM */
  int32_t smem_per_warp; /* bytes */
  int32_t slots;         /* slices per lane (1 or 2) */
  int32_t modes;         /* modes per axis the kernel was built for */
  int32_t graph;         /* 1 when the launch is a captured CUDA graph */
  int32_t kernels;       /* kernel launches per execute */
  int32_t coop_points;   /* points whose bisection several warps share (mcs_opts.coop_warps) */
  uint64_t n_points;
  uint64_t h2d_bytes; /* bytes a solve of these inputs copies host -> device */
  uint64_t d2h_bytes; /* bytes of results copied device -> host */
} mcs_plan_info;

typedef struct mcs_ctx mcs_ctx;
typedef struct mcs_plan mcs_plan;
typedef struct mcs_job mcs_job;

/* Reference defaults of timeDomainLimit: [0.05, 20] x 8, 120 revs, nonlinear, 0.45; FP64. */
void mcs_default_opts(mcs_opts* opts);

/* Message of the last failing call made by this thread ("" if none). */
const char* mcs_last_error(void);

/* Context on one CUDA device: owns a stream, device buffers and the tuned launch shapes. */
int mcs_create(mcs_ctx** ctx, int device);
int mcs_destroy(mcs_ctx* ctx);
/* The context's cudaStream_t (as void*), for callers that time or order work on it. */
void* mcs_stream(mcs_ctx* ctx);

/*
 * Batched timeDomainLimit (stabtd.js:24-32) over n_points points -- the whole Worker
 * sweep (stabworker.js:6-14) in one call.  Blocking: host inputs are copied to the
 * device, every point is solved in one persistent launch and the results are copied
 * back into out[n_points].
 */
int mcs_solve(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
              size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* opts,
              mcs_result* out);

/*
 * Several devices: the batch of mcs_solve split over the contexts ctxs[0..n_ctx) (one per
 * device, or several on one device), solved at once by one host thread per context, and the
 * results concatenated in input order into out[n_points].  Points are independent, so the
 * shards need no exchange: no peer memory, no collective.  The split is mcs_shard's.  On a
 * failure every shard still finishes; the first failing shard's status and message are
 * returned.  The multi-GPU form of the Worker's sweep (stabworker.js:6-14).
 */
int mcs_solve_multi(mcs_ctx* const* ctxs, size_t n_ctx, const mcs_setup* setups,
                    size_t n_setups, const mcs_modal* modals, size_t n_modals,
                    const mcs_point* points, size_t n_points, const mcs_opts* opts,
                    mcs_result* out);
/*
 * The split of mcs_solve_multi: each point's estimated cost (steps per trial x trials x the
 * slice evaluations a step visits, from the same FP64 preparation the solve uses) into
 * cost[i] (NULL allowed), and a longest-first greedy assignment (each point in decreasing
 * cost to the least-loaded shard, ties to the lower index) into shard_of[i] in
 * [0, n_shards).  Host arithmetic; no device needed.
 */
int mcs_shard(const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
              size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* opts,
              size_t n_shards, int32_t* shard_of, double* cost);

/*
 * Batched chatterAt (stabtd.js:14-22): one trial per entry of trials[], returning the
 * chatter index parts and the decision.  Used to replay decisions at given depths.
 */
int mcs_chatter_at(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups,
                   const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                   size_t n_points, const mcs_trial* trials, size_t n_trials,
                   const mcs_opts* opts, mcs_trial_result* out);

/*
 * Plans: the inputs of mcs_solve uploaded once and the launch captured in a CUDA graph,
 * so that repeated executions run from device-resident inputs.
 */
int mcs_plan_create(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups,
                    const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                    size_t n_points, const mcs_opts* opts, mcs_plan** plan);
int mcs_plan_execute(mcs_plan* plan); /* asynchronous on mcs_stream(ctx) */
int mcs_plan_results(mcs_plan* plan, mcs_result* out); /* waits, copies results to host */
int mcs_plan_info_get(const mcs_plan* plan, mcs_plan_info* info);
int mcs_plan_destroy(mcs_plan* plan);

/*
 * Asynchronous solve with cancellation, the Worker's job protocol (stabworker.js:7-9):
 * a cancelled job stops at the next trial boundary of each point; points not finished
 * get status MCS_ERR_CANCELLED.  out must stay valid until mcs_job_wait returns.
 */
int mcs_solve_async(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups,
                    const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                    size_t n_points, const mcs_opts* opts, mcs_result* out, mcs_job** job);
int mcs_job_poll(mcs_job* job, size_t* points_done, int* finished);
int mcs_job_cancel(mcs_job* job);
int mcs_job_wait(mcs_job* job); /* MCS_OK, or MCS_ERR_CANCELLED when cancelled */
void mcs_job_free(mcs_job* job);

/*
 * Solve without allocating: the same batched timeDomainLimit as mcs_solve, for callers
 * that must not allocate GPU memory.  Such callers are real-time loops (a machine-side
 * monitor that re-checks a few speeds per tick), where cudaMalloc/cudaFree may
 * synchronise the whole device and stall the loop, and host applications whose device
 * memory is already claimed by their own allocator or held to a fixed budget, where an
 * allocation in the middle of a run can fail with out-of-memory.  This entry point has
 * no counterpart in the reference.
 *
 * Inputs and outputs are the caller's host arrays, as for mcs_solve.  The per-point
 * parameters, the work queue and the device copy of the results live in a preallocated
 * scratch area that every GPU loading the library holds until the process exits
 * (about 0.5 MB), so a call solves at most MCS_NOALLOC_MAX_POINTS points; larger batches
 * fail with MCS_ERR_ARG.  The first call on a device looks the scratch area's device
 * address up; make that first call before any stream capture.  All calls share the area
 * and it keeps the last call's contents: the library serialises the calls per device and
 * every call, also one that fails, waits for its own copies and kernels before it
 * returns, so its calls never overlap on the GPU; work that touched the area at the same
 * time would race.  It calls no cudaMalloc, cudaFree or other allocating routine.
 */
#define MCS_NOALLOC_MAX_POINTS 1024
int mcs_solve_noalloc(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups,
                      const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                      size_t n_points, const mcs_opts* opts, mcs_result* out);

/* ------------------------------------------------------------------ schedule tuning
 * The autotuner of the schedule: no counterpart in the reference.  It captures a plan of
 * the batch for every candidate max_buckets (at most 64 candidates), runs each once
 * untimed, then times three round-robin rounds of one execution per candidate, each after
 * a write of twice the L2 size (so from a cold L2; the tuner allocates that buffer).  ms[]
 * (NULL allowed) receives each candidate's mean over the rounds and *best the fastest
 * candidate by that mean.
 * opts->max_buckets is ignored.  Results of a solve are identical for every schedule; only
 * the time changes.
 */
int mcs_tune(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
             size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* opts,
             const int32_t* candidates, size_t n_candidates, double* ms, int32_t* best);

/* ------------------------------------------------------------------ surrogate
 * A small MLP (20 -> 256 -> 256 -> 256 -> 2, SiLU, BF16 weights and activations with FP32
 * accumulation) trained on critical depths the time-domain solver itself produces.  For
 * a point it predicts mu = log critical depth and sigma (a log half-width, Gaussian NLL).
 * The guided solve either speculates the plain bisection's next levels where the
 * prediction puts them, or verifies the bracket exp(mu -+ hw) with two time-domain
 * trials, refines it by bisection and falls back to the full bisection when a
 * verification fails (mcs_guide_opts.mode).  No counterpart in the reference: it
 * accelerates timeDomainLimit (stabtd.js:24), whose plain algorithm every result is
 * checked against.
 */
#define MCS_FEATURES 20

typedef struct mcs_surrogate mcs_surrogate;

typedef struct {
  int32_t epochs;      /* passes over the training set (20) */
  int32_t batch;       /* rows per step (4096) */
  float lr;            /* Adam step (1e-3) */
  float beta1, beta2, eps;
  uint64_t seed;       /* initialisation and shuffling */
  int32_t warm;        /* nonzero: continue from the current parameters, normalisation and
                          Adam state instead of a fresh initialisation (0) */
  int32_t keep_best;   /* nonzero (with a validation set): end with the parameters of the
                          epoch of lowest validation loss (1) */
} mcs_train_opts;

/* The two guided methods.
 * MCS_GUIDE_SPECULATE (the default): after the plain first trial at a_max, the plain
 *   geometric bisection over [a_min, a_max] runs for `levels` levels, and every round runs,
 *   in lane groups beside the next midpoint, the further midpoints of the bisection tree
 *   that the predicted distribution N(mu, sigma) of the log depth makes most likely to be
 *   on the decision path.  The trials are the plain method's own, so the bracket after
 *   `levels` levels is the plain bisection's: with the configs' [0.05, 15] mm and 8 of its
 *   10 levels the guided limit lies within 1.12 % of the plain limit at every point, and a
 *   poor prediction costs rounds, never accuracy.
 * MCS_GUIDE_BRACKET: the bracket exp(mu -+ hw) is verified at both ends and refined by
 *   `refine` + extra halvings; a failed verification falls back to the full bisection. */
#define MCS_GUIDE_SPECULATE 0
#define MCS_GUIDE_BRACKET 1

typedef struct {
  float z;             /* bracket half-width hw = clamp(z * sigma, hw_min, hw_max) (log depth) */
  float hw_min, hw_max;
  float hw_direct;     /* z * sigma above this: no guess, the full bisection at once */
  int32_t refine;      /* bisection iterations inside a verified bracket (3) */
  int32_t mode;        /* MCS_GUIDE_SPECULATE (default) or MCS_GUIDE_BRACKET */
  int32_t levels;      /* speculate: bisection levels, >= 1; above opts->iters: iters (8) */
  float skip_top;      /* speculate: a point whose predicted probability of being stable at
                          a_max is below this skips the plain first trial at a_max (0, the
                          default: never).  Such a point is not reported open, so where the
                          prediction is wrong and a_max is stable its limit differs from the
                          plain one; every other point keeps the plain bracket. */
} mcs_guide_opts;

/* How each point of a guided solve was decided. */
typedef enum {
  MCS_PATH_GUIDED = 0,   /* bracket verified and refined */
  MCS_PATH_FALLBACK = 1, /* a verification failed: full bisection */
  MCS_PATH_DIRECT = 2,   /* low confidence: full bisection without verification */
  MCS_PATH_OPEN = 3      /* predicted at or past a_max and stable there */
} mcs_path;

typedef struct {
  float mu, sigma;     /* prediction: log critical depth, log half-width */
  int32_t path;        /* mcs_path */
  int32_t rounds;      /* passes of the warp over the trial loop this point took (each
                          runs one trial, or several of this point in lane groups): the
                          point's cost in time, where `trials` counts the decision path */
} mcs_guide_info;

void mcs_default_train_opts(mcs_train_opts* o);
void mcs_default_guide_opts(mcs_guide_opts* o);

/* The 20 raw (unnormalised) input features of each point, out[n * 20]: log R, N,
 * tan(helix), effective runout, log Ktc, Krc/Ktc, effective mc, log(1 + effective Ci),
 * arc start, arc end, log fz, log S, log(k zeta) and log fn of the dominant x and y modes
 * (frf.js:27), sin and cos of 2 pi fn/f_tooth for both dominant modes. */
int mcs_features(const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
                 size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* opts,
                 float* out);

/* A surrogate lives on its context's device and is destroyed before the context; destroy
 * fails with MCS_ERR_STATE while a guided plan still uses it. */
int mcs_surrogate_create(mcs_ctx* ctx, uint64_t seed, mcs_surrogate** s);
int mcs_surrogate_destroy(mcs_surrogate* s);
/* Trains on raw features X[n * 20] and targets y[n] = log critical depth; the feature
 * normalisation is taken from X.  Per-epoch mean losses go to train_loss / val_loss
 * (either may be NULL; val set optional). */
int mcs_surrogate_train(mcs_surrogate* s, const float* X, const float* y, size_t n,
                        const float* Xv, const float* yv, size_t nv, const mcs_train_opts* o,
                        float* train_loss, float* val_loss);
int mcs_surrogate_predict(mcs_surrogate* s, const float* X, size_t n, float* mu, float* sigma);
/* Mean loss and its gradient for one batch, in the parameter layout (gradient checks). */
int mcs_surrogate_grad(mcs_surrogate* s, const float* X, const float* y, size_t n, float* loss,
                       float* grad);
/* Parameters as one float array: feature mean[20], std[20], then per layer the FP32 master
 * weights W[K_pad x N_pad] (row-major, K_pad = 32 for the 20 inputs, N_pad = 16 for the 2
 * outputs, zero padding) and bias[N_pad].  get with out == NULL returns the count. */
int mcs_surrogate_get_params(mcs_surrogate* s, float* out, size_t* n_floats);
int mcs_surrogate_set_params(mcs_surrogate* s, const float* in, size_t n_floats);

/* Surrogate-guided timeDomainLimit over a batch; info (may be NULL) gets each point's
 * prediction and path.  Results are in the mcs_result layout of mcs_solve. */
int mcs_solve_guided(mcs_ctx* ctx, mcs_surrogate* s, const mcs_setup* setups, size_t n_setups,
                     const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                     size_t n_points, const mcs_opts* opts, const mcs_guide_opts* g,
                     mcs_result* out, mcs_guide_info* info);
/* The same as a device-resident plan (features, inference and solve in one CUDA graph). */
int mcs_plan_create_guided(mcs_ctx* ctx, mcs_surrogate* s, const mcs_setup* setups,
                           size_t n_setups, const mcs_modal* modals, size_t n_modals,
                           const mcs_point* points, size_t n_points, const mcs_opts* opts,
                           const mcs_guide_opts* g, mcs_plan** plan);
int mcs_plan_guide_info(mcs_plan* plan, mcs_guide_info* info);

/* ------------------------------------------------------------------ spindle speed model
 * Tool-tip modes that change with spindle speed: modesAt of src/spindle.js:64-85, which the
 * Simulator's modalNow(S) applies (src/sim.js:229-233) to give every point of a lobe sweep
 * its own modal set (src/main.js:495-496).  Host arithmetic, FP64; no device needed.
 *  - measured FRFs at several speeds (cfg.modal.speedFrfs) replace the model: the modes are
 *    interpolated linearly between the measurements (by mode order when the counts match,
 *    else the nearer measurement's), held constant outside the measured range;
 *  - else, with two_dof, the tool on a spindle mode: two tip modes of a two-mass model whose
 *    spindle spring softens with speed (spindle.js:38-53, 75-78);
 *  - else the rest modes scaled through the compliance chain 1/k = 1/k_tool + 1/k_s(S):
 *    k' = k f, fn' = fn sqrt(f), with the bearing softening k_s(S) = k_s0 / (1 + c (S/S_ref)^2),
 *    c = drop / (1 - drop) (spindle.js:18-30, 55, 79-84).
 */
typedef struct {
  double S;         /* spindle speed of the measurement [rpm] */
  mcs_modal modes;  /* tool-tip modes measured at S (ny == 0: y takes the x modes) */
} mcs_speed_frf;

typedef struct {
  mcs_modal rest;       /* modes at rest (modal.modesX/modesY, or the one {k, fn, zeta}) */
  double drop;          /* bearing-stiffness loss at s_ref, clamped to [0, 0.9]
                           (spindle.js SOFT_DEFAULT: 0.25) */
  double s_ref;         /* [rpm]; 0 reads as 30000 */
  double k_tool, k_sp;  /* compliance chain [N/mm]: tool bending, spindle/holder; a value
                           <= 0 means no chain (the rest modes at every speed) */
  int32_t two_dof;      /* 1: two tip modes from the tool (k_tool, m_tool, z_tool) on the
                           spindle mode (k_sp, m_sp, z_sp) */
  int32_t pad;
  double m_tool, m_sp;  /* [kg] */
  double z_tool, z_sp;  /* damping ratios */
} mcs_spindle;

/* The modal set at each speed S[i] into out[i] (n_frfs = 0: the model without
 * measurements).  Output sets always give ny explicitly. */
int mcs_modes_at(const mcs_spindle* spindle, const mcs_speed_frf* frfs, size_t n_frfs,
                 const double* S, size_t n_speeds, mcs_modal* out);

/* ------------------------------------------------------------------ cutting engines
 * A batch of time-domain cutting engines on one device: class CuttingEngine of
 * src/cutting.js:21-321 with every term its run() loop gives a cut -- the flutes' force law
 * with size effect, process damping, runout and a general edge profile (:115-118), the
 * axial force and the torque, the end (bottom) edges (:130-143, 215-237), a compliant thin
 * wall (:88-94, 256-264), the modal integration, the once-per-tooth samples, the decimated
 * force and position history (:288-292) and the statistics takeStats() returns.  Every
 * engine keeps its state on the device between runs, as the JS object does between run()
 * calls: the Simulator's real-time playback (Simulator.step, sim.js:351-420) configures an
 * engine for a speed, sets each substep's engagement and runs it for the substep's steps
 * (the dynamics budget of worker.js:22-32); coefficient identification (identify.js:26-40)
 * and validation (validate.js:76-100) run many rigid-tool engines in one launch.  FP64
 * arithmetic with the surface ring in float (the reference's Float32Array).  Wall samples
 * and chip events (inputs of the roughness and chip models, outside this library) are not
 * produced.  One warp simulates one engine.
 */
#define MCS_END_BINS 36
#define MCS_END_RINGS 6
#define MCS_MAX_SLICES 64
#define MCS_ENGINE_HIST 4096 /* history ring (cutting.js:28) */
#define MCS_ENGINE_TS 64     /* once-per-tooth sample ring (cutting.js:29) */

typedef struct mcs_engine mcs_engine;

/* configure(tool, modal, mat, S, fnMax) (cutting.js:39-82). */
typedef struct {
  mcs_tool tool;      /* runout and its phase as given */
  mcs_modal modal;
  double Ktc, Krc, Kac; /* shearing coefficients [N/mm^2] */
  double Kte, Kre, Kae; /* edge coefficients [N/mm] */
  double mc, Ci;      /* size-effect exponent, process-damping coefficient [N/m] */
  double S;           /* spindle speed [rpm] */
  double fn_max;      /* highest frequency to resolve besides the modes [Hz] (0) */
  int32_t nonlinear;  /* size effect and process damping (tool.nonlinear) */
  int32_t decim;      /* history every decim steps: 0 = round(spt / 40) (cutting.js:77) */
} mcs_engine_config;

/* One substep's engagement: setEngagement (:98-124), setEndEngagement (:130-143), setWork
 * (:88-94) and setWear (:85) together. */
typedef struct {
  float Hb[MCS_BINS];    /* material height at the periphery per angle bin [mm] */
  double ux, uy;         /* unit feed direction */
  double fz, tip_z, ap;  /* feed per tooth, tool tip height, engaged axial depth [mm] */
  int32_t profile;       /* 1: slice_r / slice_kap give each slice's radius [mm] and the
                            cosine of its edge angle (a general edge profile rAt) */
  int32_t wear;          /* 1: Kte / Kre below replace the material's (setWear) */
  double Kte, Kre;
  double slice_r[MCS_MAX_SLICES], slice_kap[MCS_MAX_SLICES];
  float Eb[MCS_END_BINS * MCS_END_RINGS]; /* material depth above the end face [bin][ring] */
  double fza, end_r;     /* axial feed per tooth (0: end edges idle), end-face radius [mm] */
  double ring_z[MCS_END_RINGS];  /* tip profile z at each ring's radius r_j, and at */
  double ring_zo[MCS_END_RINGS]; /*   min(end_r, r_j + dr/4) and max(0, r_j - dr/4), */
  double ring_zi[MCS_END_RINGS]; /*   dr = end_r / rings (the slope, cutting.js:135-137) */
  double wall_k, wall_m, wall_zeta; /* thin-wall mode [N/mm], [kg]; wall_k = 0: rigid */
  double wall_nx, wall_ny;          /* its unit normal */
} mcs_engagement;

/* takeStats() (cutting.js:320-323): sums since the last take, then reset. */
typedef struct {
  double n, sumF, maxF, sumFx, sumFy, sumFz, maxFz, sumT, maxT, sumX, sumY;
  double minX, maxX, minY, maxY, sumZc, wZc, sumW, maxW, sumHb, sumB, sumRb, engTeeth;
} mcs_engine_stats;

/* The state an engine carries between runs. */
typedef struct {
  double x, y, vx, vy;   /* tool position [m] and velocity [m/s] */
  double t;              /* time [s] */
  double w, wv;          /* wall deflection [m] and velocity */
  double dt;             /* step [s] */
  double run_mean_w;     /* mean wall deflection over the last run [m] */
  int32_t pr;            /* step within the revolution */
  int32_t nz;            /* slices engaged */
  int32_t steps_per_tooth, steps_per_rev, max_slices, decim;
  uint64_t step_count;
} mcs_engine_state;

int mcs_engine_create(mcs_ctx* ctx, size_t n_engines, mcs_engine** engine);
int mcs_engine_destroy(mcs_engine* engine);
/* cfg[n_engines]: a fresh engine each (the surface, modes, samples and statistics cleared). */
int mcs_engine_configure(mcs_engine* engine, const mcs_engine_config* cfg);
/* g[n_engines]: every engine's engagement for its next runs. */
int mcs_engine_set_engagement(mcs_engine* engine, const mcs_engagement* g);
/* xv[n_engines][4] = x, y [m], vx, vy [m/s]: the state set from outside (e.x = ..., the kick
 * of chatterAt); the next run moves the change into the first modes (cutting.js:163-164). */
int mcs_engine_set_state(mcs_engine* engine, const double* xv);
/* steps[n_engines] steps of each engine, all in one launch (0: that engine idles). */
int mcs_engine_run(mcs_engine* engine, const int64_t* steps);
int mcs_engine_take_stats(mcs_engine* engine, mcs_engine_stats* out);
int mcs_engine_get_state(mcs_engine* engine, mcs_engine_state* out);
/* The force and position history ring of each engine: out[e][c][MCS_ENGINE_HIST] for
 * c = Fx, Fy, Fz [N], x, y [um]; head[e] = the next write index, count[e] = samples written
 * (either may be NULL).  reset_history (validate.js:81) empties the rings. */
int mcs_engine_history(mcs_engine* engine, float* out, int32_t* head, int64_t* count);
int mcs_engine_reset_history(mcs_engine* engine);
/* chatterIndex() (cutting.js:299-318) of each engine: out[e][3] = index, amp, once. */
int mcs_engine_chatter_index(mcs_engine* engine, double* out);

/* ------------------------------------------------------------------ measurement
 * Peak rates of the context's device, measured with CUDA events on its stream: FP32 and
 * FP64 FMA issue (2 flop per FMA, every SM fully occupied) and shared-memory bandwidth
 * (16-byte loads and stores at conflict-free addresses).  The solve kernels are bounded by
 * these, not by HBM or tensor cores, so their roofline fractions are taken against these
 * figures.  No counterpart in the reference.  Takes about a second; allocates a small
 * device buffer for the call.
 */
typedef struct {
  double fp32_tflops;
  double fp64_tflops;
  double smem_tbps; /* shared memory, TB/s summed over the SMs */
} mcs_peaks;
int mcs_measure_peaks(mcs_ctx* ctx, mcs_peaks* out);

/*
 * Zero-order lobes (sld.js:23-61) read at spindle speeds (alimAt, sld.js:64-76):
 * alim[q * n_rpm + r] for query q at rpm[r]; +inf where no lobe covers the speed.
 */
int mcs_lobes_alim(mcs_ctx* ctx, const mcs_modal* modals, size_t n_modals,
                   const mcs_lobe_query* queries, size_t n_queries, const double* rpm,
                   size_t n_rpm, double* alim);

/*
 * The speed-dependent lobe diagram of the chart (Simulator.lobes, src/sim.js:262-287, with
 * LOBE_NODE and LOBE_STEP of sim.js:37): for speed-dependent dynamics the reference builds
 * one zero-order diagram per MCS_LOBE_NODE rpm over [0.8 rpm_min, 1.1 rpm_max), each with
 * the modal set at its node's centre (modesAt, see mcs_modes_at) and read (alimAt) every
 * MCS_LOBE_STEP rpm across its own node only, into one composite curve; uncovered speeds
 * read 1e3.  The chart then reads that curve per pixel (charts.js:170-185), which
 * mcs_curve_alim does.  base gives N, lobes, Ktc, Krc, the arc and the speed range (its
 * modal index is ignored).  *n_out receives the curve's length; with rpm == NULL nothing
 * else happens (a size query), else cap must hold it.  The per-node diagrams run on the
 * GPU, one CTA each.
 */
#define MCS_LOBE_NODE 1000
#define MCS_LOBE_STEP 25
int mcs_lobes_composite(mcs_ctx* ctx, const mcs_spindle* spindle, const mcs_speed_frf* frfs,
                        size_t n_frfs, const mcs_lobe_query* base, double* rpm, double* alim,
                        size_t cap, size_t* n_out);
/* alimAt (sld.js:64-76) of one lobe polyline of n_curve points at each of n speeds: the
 * interpolation on the consecutive pairs a, b with a.rpm <= S <= b.rpm, the minimum where
 * several cover S, +inf where none does.  Host arithmetic (a binary search when the speeds
 * ascend, as they do in stabilityLobes' lobes and the composite curve). */
int mcs_curve_alim(const double* curve_rpm, const double* curve_alim, size_t n_curve,
                   const double* rpm, size_t n, double* out);

#ifdef __cplusplus
}
#endif
#endif /* MCS_H_ */
