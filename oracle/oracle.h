/*
 * oracle.h -- CPU FP64 restatement of the machining simulator's time-domain chatter
 * path, used ONLY as test infrastructure: the checker for the CUDA library in tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py.  Nothing in the
 * product (libmcs.so, the mcs Python package, the Node addon) links or calls it.
 *
 * What it restates (file:line in the reference project beyond-mechanics/machinig-sim):
 *   engine.cpp  CuttingEngine configure / setEngagement / run / chatterIndex
 *               src/cutting.js:15-19, 39-82, 98-124, 146-296, 299-318
 *   stabtd.cpp  chatterAt, timeDomainLimit          src/stabtd.js:10-32
 *   sld.cpp     modeSet, frf, staticK, dominant      src/frf.js:6-27
 *               fitModes                             src/frf.js:125-144
 *               directionalCoeffs, stabilityLobes,
 *               alimAt                               src/sld.js:6-76
 *   sdm.cpp     zeroth-order semi-discretisation     test/lib/sdm.mjs:6-66
 *   tool.cpp    toolModel (uniform beam)             src/tool.js:16-32
 *               immersion                            src/identify.js:18-22
 *
 * Numbers are IEEE doubles evaluated in the reference's operation order (the build
 * uses -ffp-contract=off so no FMA fuses two roundings into one); the Float32Array
 * stores of the reference (surf, Hb, tooth samples, history) round to float here too.
 * The only arithmetic that can differ from the reference's V8 runtime is its libm
 * (Math.sin/cos/pow/tan/hypot); V8 is not available to pin that, so parity with the
 * reference is pinned by the known-answer checks its own tests and design notes give
 * (see tests/test_oracle_pins.py), not bit for bit.
 *
 * The engine also restates the terms the stability path never reaches, for the playback
 * and identification checks: the axial force and torque, end-edge forces (fza,
 * cutting.js:130-143,215-237), the thin-wall mode (:88-94,256-264), a general edge profile
 * per slice (:115-119), the full statistics and the force history.  Wall samples
 * (:269-277, roughness only) are left out.
 */
#ifndef MCS_ORACLE_H_
#define MCS_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "../include/mcs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- CuttingEngine (cutting.js:21-321) ---- */
typedef struct or_engine or_engine;

/* Engine statistics the tests read (cutting.js:280-287, takeStats). */
typedef struct {
  double n, sumF, maxF, sumFx, sumFy, sumX, sumY, engTeeth;
} or_stats;

/* Engine geometry as configured (for cross-checks with the CUDA path). */
typedef struct {
  int32_t steps_per_tooth, steps_per_rev, nz, decim, max_slices, pad;
  double dt, omega, dz;
} or_engine_info;

or_engine* or_engine_new(void);
void or_engine_free(or_engine* e);
/* configure(tool, modal, mat, S, fnMax) (cutting.js:39-82) with the tool's nonlinear
 * flag; spt_override / slices_override > 0 replace the step and slice rules. */
void or_engine_configure(or_engine* e, const mcs_tool* tool, int nonlinear,
                         const mcs_modal* modal, const mcs_material* mat, double S,
                         double fn_max, int spt_override, int slices_override);
/* The 180-bin material-height map Hb (Float32Array, cutting.js:23), filled by callers. */
float* or_engine_hb(or_engine* e);
/* setEngagement(u, fz, tipZ, ap) (cutting.js:98-124). */
void or_engine_set_engagement(or_engine* e, double ux, double uy, double fz, double tipZ,
                              double ap);
/* Assign the externally visible state (e.g. the test kick e.vx = 0.01). */
void or_engine_set_state(or_engine* e, double x, double y, double vx, double vy);
/* run(nSteps) (cutting.js:146-296). */
void or_engine_run(or_engine* e, int64_t n_steps);
/* chatterIndex() (cutting.js:299-318): out = {index, amp (sAll), once (sOnce)}. */
void or_engine_chatter_index(const or_engine* e, double out[3]);
/* takeStats() (cutting.js:320). */
void or_engine_take_stats(or_engine* e, or_stats* out);
/* Volumes of the chip events so far, oldest first (cutting.js:238-242). */
int or_engine_chip_vols(const or_engine* e, double* out, int cap);
void or_engine_get_info(const or_engine* e, or_engine_info* out);
/* The rest of the engine's cutting terms, for the playback / identification oracle: the
 * axial coefficients, setWear, the end-face map Eb (36 x 6 floats, filled by callers),
 * setEndEngagement with the tip profile sampled at the rings, setWork (k <= 0: none), a
 * general edge profile per slice, the full takeStats() and the force/position history. */
void or_engine_set_axial(or_engine* e, double Kac, double Kae);
void or_engine_set_wear(or_engine* e, int on, double Kte, double Kre);
float* or_engine_eb(or_engine* e);
void or_engine_set_end(or_engine* e, double fza, double rOut, const double* z_at,
                       const double* z_out, const double* z_in);
void or_engine_set_work(or_engine* e, double k, double m, double zeta, double nx, double ny);
void or_engine_set_engagement_profile(or_engine* e, double ux, double uy, double fz,
                                      double tipZ, double ap, const double* prof_r,
                                      const double* prof_kap);
void or_engine_take_stats_full(or_engine* e, mcs_engine_stats* out);
void or_engine_history(const or_engine* e, float* out, int32_t* head, int64_t* count);
void or_engine_reset_history(or_engine* e);
/* e.decim = decim (validate.js:80 samples every step). */
void or_engine_set_decim(or_engine* e, int decim);

/* ---- stabtd.js ---- */
/* One chatterAt trial (stabtd.js:14-22) with the option set of mcs_opts. */
void or_chatter_at(const mcs_setup* setup, const mcs_modal* modal, double S, double ap,
                   const mcs_opts* opts, mcs_trial_result* out);

/* Trial record of a bisection: depth, chatterIndex parts and decision. */
typedef struct {
  double ap, index, once, amp;
  int32_t chatter, pad;
} or_trace_entry;

/* timeDomainLimit (stabtd.js:24-32).  trace (may be NULL) receives up to iters+1 trials. */
void or_time_domain_limit(const mcs_setup* setup, const mcs_modal* modal, double S,
                          const mcs_opts* opts, mcs_result* out, or_trace_entry* trace);

/* Thread-pool drivers over batches (points index setups/modals as in mcs_solve).
 * traces: n_points * (iters+1) entries or NULL.  nthreads <= 0: all hardware threads. */
void or_solve_batch(const mcs_setup* setups, const mcs_modal* modals, const mcs_point* points,
                    size_t n_points, const mcs_opts* opts, mcs_result* out,
                    or_trace_entry* traces, int nthreads);
void or_chatter_batch(const mcs_setup* setups, const mcs_modal* modals,
                      const mcs_point* points, const mcs_trial* trials, size_t n_trials,
                      const mcs_opts* opts, mcs_trial_result* out, int nthreads);

/* ---- frf.js / sld.js ---- */
void or_frf(const mcs_mode* modes, int n, double f, double out[2]);
double or_static_k(const mcs_mode* modes, int n);
int or_dominant(const mcs_mode* modes, int n);
/* directionalCoeffs: out = {xx, xy, yx, yy}. */
void or_directional_coeffs(double Kr, double phi_st, double phi_ex, double out[4]);
/* stabilityLobes: lobes are written one after another into rpm/alim (capacity cap);
 * lobe_len[j] gets the length of lobe j.  Returns the number of lobes, or -1 when cap
 * is too small. */
int or_stability_lobes(const mcs_lobe_query* q, const mcs_modal* modal, double* rpm,
                       double* alim, int32_t* lobe_len, int cap);
/* alimAt over lobes laid out as or_stability_lobes writes them. */
double or_alim_at(int n_lobes, const int32_t* lobe_len, const double* rpm, const double* alim,
                  double at_rpm);
/* stabilityLobes + alimAt for many queries and speeds: out[q * n_rpm + r]. */
void or_lobes_alim(const mcs_modal* modals, const mcs_lobe_query* queries, size_t n_queries,
                   const double* rpm, size_t n_rpm, double* out);
/* fitModes (frf.js:125-144) on a sampled FRF G = re + i im [mm/N]; returns modes written. */
int or_fit_modes(const double* f, const double* re, const double* im, int n, int max_modes,
                 mcs_mode* out);

/* ---- test/lib/sdm.mjs ---- */
typedef struct {
  double m, k, zeta, Kt, Kn;
  int32_t N, steps;
  double phi_st, phi_ex, rpm;
} or_sdm_params;
double or_sdm_rho(const or_sdm_params* p, double a);
double or_sdm_limit(const or_sdm_params* p, double a_max);

/* ---- tool.js / identify.js ---- */
/* toolModel of a uniform beam: out = {k [N/mm], fn [Hz], kTool [N/mm], mEff [kg]}. */
void or_tool_model(double D, double stickout, double k_spindle, double m_holder, double out[4]);
// spindle.js modesAt at each speed (spindle.cpp)
void or_modes_at(const mcs_spindle* sp, const mcs_speed_frf* frfs, size_t n_frfs,
                 const double* S, size_t n, mcs_modal* out);
/* immersion(mode, ae, D): mode 0 slot, 1 down, 2 up; out = {phiSt, phiEx}. */
void or_immersion(int mode, double ae, double D, double out[2]);

#ifdef __cplusplus
}
#endif
#endif
