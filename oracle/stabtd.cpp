// Oracle (test infrastructure only): chatterAt and timeDomainLimit of src/stabtd.js:10-32
// on top of the engine restatement, plus std::thread pool drivers for batches (the
// multi-core analogue of the stability Worker's sequential loop, src/stabworker.js:6-14).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

constexpr double kPi = 3.141592653589793;

// The engine configuration chatterAt builds (stabtd.js:15-20) and the trial itself.
void trial(const mcs_setup* setup, const mcs_modal* modal, double S, double ap,
           const mcs_opts* o, double out_idx[3]) {
  or_engine* e = or_engine_new();
  mcs_tool tool = setup->tool;
  tool.flute_len = std::max(setup->tool.flute_len, ap + 1);
  if (!o->honor_runout) {  // chatterAt runs without runout (stabtd.js:7-9,16)
    tool.runout = 0;
    tool.runout_phase = 0;
  }
  or_engine_configure(e, &tool, o->nonlinear, modal, &setup->mat, S, 0, o->steps_per_tooth,
                      o->slices);
  float* Hb = or_engine_hb(e);
  for (int b = 0; b < MCS_BINS; b++) {
    const double phi = (b + 0.5) / MCS_BINS * 2 * kPi;
    Hb[b] = (phi >= setup->arc_st && phi <= setup->arc_ex) ? 0.f : -1e3f;
  }
  or_engine_set_engagement(e, 1, 0, setup->fz, -ap, ap);
  or_engine_set_state(e, 0, 0, 0.01, 0);  // a small kick
  or_engine_info info;
  or_engine_get_info(e, &info);
  or_engine_run(e, (int64_t)info.steps_per_tooth * tool.N * o->revs);
  or_engine_chatter_index(e, out_idx);
  or_engine_free(e);
}

}  // namespace

extern "C" {

void or_chatter_at(const mcs_setup* setup, const mcs_modal* modal, double S, double ap,
                   const mcs_opts* opts, mcs_trial_result* out) {
  double ci[3];
  trial(setup, modal, S, ap, opts, ci);
  out->index = ci[0];
  out->amp = ci[1];
  out->once = ci[2];
  out->chatter = ci[0] > opts->chatter_idx;
  out->status = MCS_OK;
}

void or_time_domain_limit(const mcs_setup* setup, const mcs_modal* modal, double S,
                          const mcs_opts* o, mcs_result* out, or_trace_entry* trace) {
  int nt = 0;
  auto chatter = [&](double ap) {
    mcs_trial_result r;
    or_chatter_at(setup, modal, S, ap, o, &r);
    if (trace) {
      trace[nt].ap = ap;
      trace[nt].index = r.index;
      trace[nt].once = r.once;
      trace[nt].amp = r.amp;
      trace[nt].chatter = r.chatter;
      trace[nt].pad = 0;
    }
    nt++;
    return r.chatter != 0;
  };
  out->status = MCS_OK;
  out->engaged = 0;
  out->evals = 0;
  out->steps_per_tooth = 0;
  if (!chatter(o->a_max)) {
    out->alim = o->a_max;
    out->lo = o->a_max;
    out->hi = std::numeric_limits<double>::infinity();
    out->open = 1;
    out->trials = nt;
    return;
  }
  double lo = o->a_min, hi = o->a_max;
  for (int i = 0; i < o->iters; i++) {
    const double m = std::sqrt(lo * hi);
    if (chatter(m))
      hi = m;
    else
      lo = m;
  }
  out->alim = std::sqrt(lo * hi);
  out->lo = lo;
  out->hi = hi;
  out->open = 0;
  out->trials = nt;
}

void or_solve_batch(const mcs_setup* setups, const mcs_modal* modals, const mcs_point* points,
                    size_t n_points, const mcs_opts* opts, mcs_result* out,
                    or_trace_entry* traces, int nthreads) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = (int)std::min<size_t>((size_t)nthreads, std::max<size_t>(n_points, 1));
  std::atomic<size_t> next{0};
  const int per = opts->iters + 1;
  auto work = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= n_points) break;
      const mcs_point& p = points[i];
      or_time_domain_limit(&setups[p.setup], &modals[p.modal], p.S, opts, &out[i],
                           traces ? traces + i * per : nullptr);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthreads; t++) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

void or_chatter_batch(const mcs_setup* setups, const mcs_modal* modals,
                      const mcs_point* points, const mcs_trial* trials, size_t n_trials,
                      const mcs_opts* opts, mcs_trial_result* out, int nthreads) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = (int)std::min<size_t>((size_t)nthreads, std::max<size_t>(n_trials, 1));
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= n_trials) break;
      const mcs_point& p = points[trials[i].point];
      or_chatter_at(&setups[p.setup], &modals[p.modal], p.S, trials[i].ap, opts, &out[i]);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthreads; t++) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

}  // extern "C"
