// C ABI of libmcs.so (include/mcs.h): input validation, per-point preparation on the
// host (the FP64 derivations of CuttingEngine.configure, src/cutting.js:39-82), work
// ordering and bucketing, CUDA-graph plans, blocking and asynchronous solves.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <numeric>
#include <queue>
#include <string>
#include <thread>
#include <vector>

#include "mcs_internal.h"

using namespace mcs;

namespace {
thread_local std::string g_last_error;
}  // namespace

int mcs::fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

namespace {

#define MCS_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(MCS_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));         \
  } while (0)

constexpr double kPi = 3.141592653589793;
constexpr int kMaxBuckets = MCS_MAX_BUCKETS;
constexpr int kDefaultBuckets = 16;

inline bool is_finite(double v) { return std::isfinite(v); }

// ------------------------------------------------------------------ validation
int check_inputs(const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
                 size_t n_modals, const mcs_point* points, size_t n_points,
                 const mcs_opts* o) {
  if (!o) return fail(MCS_ERR_ARG, "opts is NULL");
  if (n_points && (!setups || !modals || !points))
    return fail(MCS_ERR_ARG, "NULL input array");
  if (n_points > (size_t)std::numeric_limits<int32_t>::max())
    return fail(MCS_ERR_ARG, "too many points (%zu)", n_points);
  if (!(is_finite(o->a_min) && is_finite(o->a_max) && o->a_min > 0 && o->a_max >= o->a_min))
    return fail(MCS_ERR_ARG, "bisection range must satisfy 0 < a_min <= a_max");
  if (o->iters < 0 || o->iters > 60) return fail(MCS_ERR_ARG, "iters out of range [0, 60]");
  if (o->revs < 1 || o->revs > 1000000) return fail(MCS_ERR_ARG, "revs out of range");
  if (o->steps_per_tooth < 0 || o->steps_per_tooth > 10000000)
    return fail(MCS_ERR_ARG, "steps_per_tooth out of range");
  if (o->slices < 0) return fail(MCS_ERR_ARG, "slices must be >= 0");
  if (o->slices > kMaxSlots * kWarp)
    return fail(MCS_ERR_UNSUPPORTED, "at most %d slices are supported", kMaxSlots * kWarp);
  if (!is_finite(o->chatter_idx)) return fail(MCS_ERR_ARG, "chatter_idx is not finite");
  if (o->precision != MCS_FP32 && o->precision != MCS_FP64)
    return fail(MCS_ERR_ARG, "precision must be MCS_FP32 or MCS_FP64");
  if (o->max_buckets < 0 || o->max_buckets > kMaxBuckets)
    return fail(MCS_ERR_ARG, "max_buckets out of range [0, %d]", kMaxBuckets);
  if (o->serial_trials != 0 && o->serial_trials != 1)
    return fail(MCS_ERR_ARG, "serial_trials must be 0 or 1");
  if (o->coop_warps < 0 || o->coop_warps > kCoopMaxWarpsHost)
    return fail(MCS_ERR_ARG, "coop_warps out of range [0, %d]", kCoopMaxWarpsHost);
  if (o->coop_points < 0) return fail(MCS_ERR_ARG, "coop_points must be >= 0");
  for (size_t i = 0; i < n_setups; i++) {
    const mcs_setup& s = setups[i];
    const mcs_tool& t = s.tool;
    if (t.N < 1 || t.N > kMaxTeeth)
      return fail(MCS_ERR_ARG, "setup %zu: N must be in [1, %d]", i, kMaxTeeth);
    if (t.type != MCS_TOOL_FLAT && t.type != MCS_TOOL_BALL)
      return fail(MCS_ERR_ARG, "setup %zu: unknown tool type", i);
    if (!(is_finite(t.R) && t.R > 0)) return fail(MCS_ERR_ARG, "setup %zu: R must be > 0", i);
    if (!(is_finite(t.helix_deg) && std::fabs(t.helix_deg) < 89))
      return fail(MCS_ERR_ARG, "setup %zu: helix out of range", i);
    if (!(is_finite(t.flute_len) && t.flute_len > 0))
      return fail(MCS_ERR_ARG, "setup %zu: flute_len must be > 0", i);
    if (!(is_finite(t.runout) && is_finite(t.runout_phase)))
      return fail(MCS_ERR_ARG, "setup %zu: runout not finite", i);
    const mcs_material& m = s.mat;
    if (!(is_finite(m.Ktc) && is_finite(m.Krc) && is_finite(m.Kte) && is_finite(m.Kre) && is_finite(m.mc) &&
          is_finite(m.Ci) && m.mc >= 0 && m.Ci >= 0))
      return fail(MCS_ERR_ARG, "setup %zu: material coefficients invalid", i);
    if (!(is_finite(s.fz) && s.fz > 0)) return fail(MCS_ERR_ARG, "setup %zu: fz must be > 0", i);
    if (!(is_finite(s.arc_st) && is_finite(s.arc_ex)))
      return fail(MCS_ERR_ARG, "setup %zu: arc not finite", i);
  }
  for (size_t i = 0; i < n_modals; i++) {
    const mcs_modal& md = modals[i];
    if (md.nx < 1 || md.nx > kMaxModes || md.ny < 0 || md.ny > kMaxModes)
      return fail(MCS_ERR_ARG, "modal %zu: 1 <= nx <= %d and 0 <= ny <= %d", i, kMaxModes,
                  kMaxModes);
    for (int a = 0; a < 2; a++) {
      const int cnt = a == 0 ? md.nx : md.ny;
      const mcs_mode* ms = a == 0 ? md.x : md.y;
      for (int j = 0; j < cnt; j++)
        if (!(is_finite(ms[j].k) && ms[j].k > 0 && is_finite(ms[j].fn) && ms[j].fn > 0 &&
              is_finite(ms[j].zeta) && ms[j].zeta >= 0))
          return fail(MCS_ERR_ARG, "modal %zu: mode %d needs k > 0, fn > 0, zeta >= 0", i, j);
    }
  }
  for (size_t i = 0; i < n_points; i++) {
    const mcs_point& p = points[i];
    if (p.setup >= n_setups) return fail(MCS_ERR_ARG, "point %zu: setup index out of range", i);
    if (p.modal >= n_modals) return fail(MCS_ERR_ARG, "point %zu: modal index out of range", i);
    if (!(is_finite(p.S) && p.S > 0)) return fail(MCS_ERR_ARG, "point %zu: S must be > 0", i);
  }
  return MCS_OK;
}

// ------------------------------------------------------------------ preparation
// Slices a trial at depth ap uses (setEngagement with chatterAt's fluteLen).
int slices_at(double ap, double flute_len, int override_n) {
  if (ap <= 0) return 0;
  if (override_n > 0) return override_n;
  const double flute = std::max(flute_len, ap + 1.0);
  const double dz = std::max(0.25, flute / 48.0);
  const int maxs = (int)std::ceil(flute / dz);
  return std::min(maxs, (int)std::ceil(ap / dz));
}

struct Prepared {
  PointParams pp;
  double cost;
  int modes;  // max modes per axis
  int nl;     // size effect or process damping present
};

int prepare_point(const mcs_setup& st, const mcs_modal& md, double S_in, const mcs_opts& o,
                  double ap_max, Prepared& out) {
  PointParams& P = out.pp;
  std::memset(&P, 0, sizeof(P));
  const mcs_tool& t = st.tool;
  const int N = t.N;
  const double S = std::max(100.0, S_in);
  const double omega = S * 2 * kPi / 60;
  const double Ttooth = 60 / (S * N);
  const int nx = md.nx, ny = md.ny > 0 ? md.ny : md.nx;
  const mcs_mode* xm = md.x;
  const mcs_mode* ym = md.ny > 0 ? md.y : md.x;
  double fTop = -INFINITY;
  for (int j = 0; j < nx; j++) fTop = std::max(fTop, xm[j].fn);
  for (int j = 0; j < ny; j++) fTop = std::max(fTop, ym[j].fn);
  // steps per tooth period: 24 per period of the highest mode, at least 48 (cutting.js:50)
  double sptd = o.steps_per_tooth > 0 ? (double)o.steps_per_tooth
                                      : std::max(48.0, std::ceil(Ttooth * fTop * 24));
  const double nsteps_d = sptd * N * (double)o.revs;
  if (sptd * N > 1e7 || nsteps_d >= 2147483647.0)
    return fail(MCS_ERR_UNSUPPORTED, "trial of %.0f steps is too long for the kernels", nsteps_d);
  const int spt = (int)sptd;
  const double dt = Ttooth / spt;
  P.omega = omega;
  P.dphi = omega * dt;
  P.R = t.R;
  P.tanB = std::tan(t.helix_deg * kPi / 180);
  P.flute_len = t.flute_len;
  P.Ci = o.nonlinear ? st.mat.Ci : 0.0;
  P.fz = st.fz;
  P.hmax = std::max(0.1, 3 * st.fz);
  P.Ktc = st.mat.Ktc;
  P.Krc = st.mat.Krc;
  P.Kte = st.mat.Kte;
  P.Kre = st.mat.Kre;
  P.mc = o.nonlinear ? st.mat.mc : 0.0;
  P.dt = dt;
  // runout offsets delta_i = e cos(2 pi i / N - gamma) (cutting.js:44); chatterAt uses 0
  for (int i = 0; i < N; i++)
    P.dR[i] = o.honor_runout ? t.runout * std::cos(2 * kPi * i / N - t.runout_phase) : 0.0;
  // modes: k [N/m], m = k / (2 pi fn)^2, c = 2 zeta sqrt(k m) (cutting.js:54-59)
  for (int a = 0; a < 2; a++) {
    const int cnt = a == 0 ? nx : ny;
    const mcs_mode* ms = a == 0 ? xm : ym;
    for (int j = 0; j < cnt; j++) {
      const double k = ms[j].k * 1e3;
      const double w = 2 * kPi * ms[j].fn;
      const double m = k / (w * w);
      const double c = 2 * ms[j].zeta * std::sqrt(k * m);
      P.mk[a][j] = k;
      P.mcd[a][j] = c;
      P.ma[a][j] = dt / m;
    }
  }
  out.modes = std::max(nx, ny);
  out.nl = (P.mc != 0.0 || P.Ci != 0.0) ? 1 : 0;
  P.N = N;
  P.spt = spt;
  P.spr = N * spt;
  P.decim = (int)std::max(1.0, std::floor(spt / 40.0 + 0.5));
  P.nsteps = (int)nsteps_d;
  P.type = t.type;
  P.slices_override = o.slices;
  // engaged bins of the static map chatterAt builds (stabtd.js:17): bin b is in the
  // arc when its centre (b + 0.5)/180*2pi lies in [arc_st, arc_ex]
  int b0 = -1, b1 = -1;
  for (int b = 0; b < MCS_BINS; b++) {
    const double phi = (b + 0.5) / MCS_BINS * 2 * kPi;
    if (phi >= st.arc_st && phi <= st.arc_ex) {
      if (b0 < 0) b0 = b;
      b1 = b;
    }
  }
  const double binScale = MCS_BINS / (2 * kPi);
  P.empty = b0 < 0 ? 1 : 0;
  if (!P.empty) {
    P.phi_lo = b0 / binScale;
    // sin(phi) <= 0 is out of cut (cutting.js:190): nothing at or past pi
    P.phi_hi = std::min((b1 + 1) / binScale, kPi);
    P.excl_zero = b0 == 0 ? 1 : 0;
    if (P.phi_hi <= P.phi_lo) P.empty = 1;
  }
  const double span = P.empty ? 0.0 : P.phi_hi - P.phi_lo;
  const int lmax = P.empty ? 1 : (int)std::floor(span / P.dphi) + 2;
  P.lpad = std::min(lmax, P.spr) | 1;
  P.nz_max = slices_at(ap_max, t.flute_len, o.slices);
  if (P.nz_max > kMaxSlots * kWarp)
    return fail(MCS_ERR_UNSUPPORTED, "%d slices exceed the %d the kernels support", P.nz_max,
                kMaxSlots * kWarp);
  // chatter-index windows (cutting.js:301,310): the last n tooth samples and the last
  // m = round(n spt / decim) history samples
  const long long C = (long long)N * o.revs;
  P.ts_n = (int)std::min<long long>(C, 24);
  P.ts_c0 = (int)(C - P.ts_n);
  const long long H = (long long)P.nsteps / P.decim;
  P.hist_m = (int)std::min<long long>(H, (long long)std::floor((double)P.ts_n * spt / P.decim + 0.5));
  P.hist_h0 = (int)(H - P.hist_m);
  // trials of one point can share a warp in lane groups when their slice counts vary with
  // depth (the reference slice rule) or are small; the ring then has a row per lane
  P.groups = (!o.serial_trials && (o.slices == 0 || o.slices <= 16)) ? kMaxGroups : 1;
  P.ring_rows = P.groups > 1 ? std::max(P.nz_max, kWarp) : P.nz_max;
  const long long smem =
      warp_smem(P.spr, o.precision == MCS_FP64, P.ring_rows, P.lpad, P.groups);
  if (smem > kMaxSmemPerWarp)
    return fail(MCS_ERR_UNSUPPORTED,
                "point needs %lld bytes of shared memory (spr %d, %d slices): above %d", smem,
                P.spr, P.nz_max, kMaxSmemPerWarp);
  P.smem_bytes = (int)smem;
  // relative cost for ordering: steps x (visited teeth x slots + fixed per-step work)
  const double lag_span = std::fabs(ap_max * P.tanB / P.R);
  const double act = std::min(1.0, (span + lag_span) / (2 * kPi) + 1.0 / N);
  const int slots = (P.nz_max + kWarp - 1) / kWarp;
  out.cost = (double)P.nsteps * (o.iters + 1) * (24.0 + 40.0 * N * std::max(1, slots) * act);
  return MCS_OK;
}

int slots_for(int nz) { return nz <= kWarp ? 1 : 2; }

// The surrogate's 20 raw input features of a point (mcs_features in include/mcs.h).
void point_features(const mcs_setup& st, const mcs_modal& md, double S_in, const mcs_opts& o,
                    float* f) {
  const mcs_tool& t = st.tool;
  const mcs_material& m = st.mat;
  const int nx = md.nx, ny = md.ny > 0 ? md.ny : md.nx;
  const mcs_mode* xm = md.x;
  const mcs_mode* ym = md.ny > 0 ? md.y : md.x;
  // dominant mode: the lowest k * zeta, the first of equals (frf.js:27)
  auto dominant = [](const mcs_mode* ms, int n) {
    int a = 0;
    for (int i = 1; i < n; i++)
      if (ms[i].k * ms[i].zeta < ms[a].k * ms[a].zeta) a = i;
    return ms[a];
  };
  const mcs_mode dx = dominant(xm, nx), dy = dominant(ym, ny);
  const double S = std::max(100.0, S_in);
  const double ft = S * t.N / 60.0;  // tooth-passing frequency [Hz]
  const double two_pi = 2 * kPi;
  f[0] = (float)std::log(t.R);
  f[1] = (float)t.N;
  f[2] = (float)std::tan(t.helix_deg * kPi / 180);
  f[3] = (float)(o.honor_runout ? t.runout : 0.0);
  f[4] = (float)std::log(std::max(m.Ktc, 1e-9));
  f[5] = (float)(m.Krc / std::max(m.Ktc, 1e-9));
  f[6] = (float)(o.nonlinear ? m.mc : 0.0);
  f[7] = (float)std::log1p(o.nonlinear ? m.Ci : 0.0);
  f[8] = (float)st.arc_st;
  f[9] = (float)st.arc_ex;
  f[10] = (float)std::log(st.fz);
  f[11] = (float)std::log(S);
  f[12] = (float)std::log(dx.k * std::max(dx.zeta, 1e-6));
  f[13] = (float)std::log(dx.fn);
  f[14] = (float)std::log(dy.k * std::max(dy.zeta, 1e-6));
  f[15] = (float)std::log(dy.fn);
  f[16] = (float)std::sin(two_pi * dx.fn / ft);
  f[17] = (float)std::cos(two_pi * dx.fn / ft);
  f[18] = (float)std::sin(two_pi * dy.fn / ft);
  f[19] = (float)std::cos(two_pi * dy.fn / ft);
}

// ------------------------------------------------------------------ device buffers
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return MCS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      p = nullptr;
      return fail(e == cudaErrorMemoryAllocation ? MCS_ERR_NOMEM : MCS_ERR_CUDA,
                  "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    cap = want;
    return MCS_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct Bucket {
  KernelShape shape;
  int smem = 0;
  int grid = 0;
  int offset = 0;  // into the order array
  int count = 0;
  int blocks_per_sm = 0;
};

}  // namespace

struct mcs_ctx {
  int device = 0;
  mcs_plan* solve_scratch = nullptr;   // mcs_solve's plan, reused so calls allocate nothing new
  mcs_plan* guided_scratch = nullptr;  // mcs_solve_guided's plan, likewise
  int sms = 0;
  int prio_low = 0, prio_high = 0;  // stream priority range (lower value = scheduled first)
  cudaStream_t stream = nullptr;
  cudaStream_t aux[kMaxBuckets] = {};  // one per bucket for direct (uncaptured) calls
  cudaStream_t side = nullptr;  // progress reads and cancellation while a job runs
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kMaxBuckets] = {};
  std::mutex mu;
  void* pinned = nullptr;  // upload staging (page-locked), grown on demand
  size_t pinned_cap = 0;
};

int mcs::ctx_device(mcs_ctx* c) { return c->device; }
cudaStream_t mcs::ctx_stream(mcs_ctx* c) { return c->stream; }

struct mcs_plan {
  mcs_ctx* ctx = nullptr;
  size_t n = 0;
  bool trials = false;
  // surrogate guidance (guided plans)
  mcs_surrogate* sur = nullptr;
  mcs_guide_opts gopts{};
  double a_max = 0.0;  // the bisection's upper end (the guide's skip_top test)
  DevBuf feat, gmu, gsigma, guide, ginfo;
  std::vector<Bucket> buckets;
  DevBuf params, order, results, queues, items;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int max_modes = 1;
  int max_slots = 1;
  bool executed = false;
};

struct mcs_job {
  mcs_plan* plan = nullptr;
  mcs_result* out = nullptr;
  mcs_result* staging = nullptr;  // pinned
  DevBuf cancel, progress;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool waited = false;
};

namespace {

// The multi-warp head of a plain solve: the `head` costliest points (in cost order) that
// do not speculate in lane groups already, each on the widest block whose rings fit in
// shared memory (`coop_warps`, else 4, else 3 warps; a point that fits none stays on the
// one-warp path).  One bucket per width, the one holding the costliest point first; the
// points of all of them are appended to `members` in bucket order.
void coop_head_buckets(const std::vector<double>& cost, const std::vector<int>& slots,
                       const std::vector<int>& modes, const std::vector<int>& nls,
                       const std::vector<int>& grps, const std::vector<PointParams>& pp,
                       int fp64, int coop_warps, int head, std::vector<int32_t>& members,
                       std::vector<Bucket>& heads) {
  const size_t n = cost.size();
  std::vector<int32_t> byc(n);
  std::iota(byc.begin(), byc.end(), 0);
  std::stable_sort(byc.begin(), byc.end(), [&](int a, int c) { return cost[a] > cost[c]; });
  members.clear();
  heads.clear();
  const int widths[3] = {coop_warps, std::min(coop_warps, 4), std::min(coop_warps, 3)};
  std::vector<int32_t> part[3];
  int taken = 0;
  for (int32_t q : byc) {
    if (taken >= head) break;
    // lane groups speculate without extra warps, but only while a trial's slices fit in a
    // fraction of the warp: points whose deepest trials need more than half of it run
    // their deep levels serially there, and take the multi-warp path like the others
    if (grps[q] && pp[q].nz_max <= kWarp / 2) continue;
    for (int k = 0; k < 3; k++) {
      if (k > 0 && widths[k] == widths[k - 1]) continue;
      const int cs = coop_smem(pp[q].spr, fp64 != 0, pp[q].ring_rows, pp[q].lpad, widths[k]);
      if (((cs + 15) & ~15) <= kCoopSmemLimit) {
        part[k].push_back(q);
        taken++;
        break;
      }
    }
  }
  // buckets in the order of their costliest point (each part is in cost order)
  int ord[3] = {0, 1, 2};
  auto rank = [&](int k) -> double { return part[k].empty() ? -1.0 : cost[part[k][0]]; };
  std::stable_sort(ord, ord + 3, [&](int a, int b) { return rank(a) > rank(b); });
  for (int k : ord) {
    if (part[k].empty()) continue;
    int sl = 1, nm = 1, nl = 0, cs = 0;
    for (int32_t q : part[k]) {
      sl = std::max(sl, slots[q]);
      nm = std::max(nm, modes[q]);
      nl = std::max(nl, nls[q]);
      cs = std::max(cs, coop_smem(pp[q].spr, fp64 != 0, pp[q].ring_rows, pp[q].lpad,
                                  widths[k]));
    }
    Bucket b;
    b.shape = KernelShape{sl, nm, fp64, nl, 0};
    b.shape.coop = widths[k];
    b.smem = (cs + 15) & ~15;
    int cb = 0;
    if (occupancy_solve(b.shape, b.smem, &cb) != 0 || cb < 1) continue;  // one-warp path
    b.offset = (int)members.size();
    b.count = (int)part[k].size();
    members.insert(members.end(), part[k].begin(), part[k].end());
    heads.push_back(b);
  }
}

// The library's rule for the multi-warp head: the points whose own serial bisection costs
// more than the batch's share of one resident warp, i.e. the points that would still run
// after the device has finished everything else.  The share takes a resident warp to do
// 0.65 of the work of a warp alone on its SM (the 4096-speed sweep, bound by its total
// work: 8 resident FP64 warps per SM did that of 5.8 lone warps, 13 FP32 ones that of 7.3).
int coop_auto_head(mcs_ctx* ctx, const std::vector<int>& smem, const std::vector<double>& cost,
                   const std::vector<int>& slots, const std::vector<int>& modes,
                   const std::vector<int>& nls, const std::vector<int>& grps, int fp64) {
  const size_t n = cost.size();
  if (n == 0) return 0;
  std::vector<int32_t> byc(n);
  std::iota(byc.begin(), byc.end(), 0);
  std::stable_sort(byc.begin(), byc.end(), [&](int a, int c) { return cost[a] > cost[c]; });
  const int32_t m = byc[n / 2];  // a typical point's residency
  KernelShape ks{slots[m], modes[m], fp64, nls[m], grps[m]};
  int bps = 0;
  if (occupancy_solve(ks, (smem[m] + 15) & ~15, &bps) != 0 || bps < 1) bps = 1;
  double total = 0.0;
  for (double c : cost) total += c;
  const double share = total / ((double)ctx->sms * std::max(1.0, 0.65 * bps));
  int head = 0;
  while (head < (int)n && head < 2 * ctx->sms && cost[byc[head]] > share) head++;
  return head;
}

// Orders the work items by cost (largest first) and groups them into buckets of similar
// shared-memory need, each launched as its own persistent grid.
//
// Multi-warp bisection (plain solves): the `coop_head` costliest points run each on
// `coop_warps` warps of one block, as a bucket of their own ahead of the others (the
// latency tail of the slowest points; see solve_coop_kernel and coop_head_bucket).  pp
// (NULL for trial batches) gives the per-point sizes the multi-warp shared memory follows
// from.
int make_buckets(mcs_ctx* ctx, const std::vector<int>& smem, const std::vector<double>& cost,
                 const std::vector<int>& slots, const std::vector<int>& modes,
                 const std::vector<int>& nls, const std::vector<int>& grps, bool trials,
                 int fp64, int max_buckets,
                 std::vector<int32_t>& order, std::vector<Bucket>& buckets,
                 const std::vector<PointParams>* pp = nullptr, int coop_warps = 1,
                 int coop_head = 0) {
  int nbmax = max_buckets > 0 ? std::min(max_buckets, kMaxBuckets) : kDefaultBuckets;
  const size_t n_all = smem.size();
  buckets.clear();
  order.clear();
  order.reserve(n_all);
  if (n_all == 0) return MCS_OK;
  bool any_head = false;  // a multi-warp head leads the batch
  // resident blocks per SM and grid of a bucket, which then joins the list
  auto place = [&](Bucket& b) -> int {
    int bps = 0;
    const int rc = trials ? occupancy_trials(b.shape, b.smem, &bps)
                          : occupancy_solve(b.shape, b.smem, &bps);
    if (rc != 0)
      return fail(MCS_ERR_CUDA, "occupancy query failed: %s",
                  cudaGetErrorString((cudaError_t)rc));
    if (bps < 1)
      return fail(MCS_ERR_UNSUPPORTED, "a %d-byte warp does not fit on an SM", b.smem);
    // An FP64 linear bucket takes the kernel held to more resident warps when its shared
    // memory lets them reside: a warp of it runs at 0.87 of the default's speed (spilled
    // words), and the SM's rate grows with its resident warps (measured on one B200:
    // 148 x k uniform points, k = 1 ... 8 warps per SM in proportion), so it pays from
    // 10 resident warps against the default's 8.  Only in a batch bound by its total work:
    // beside a multi-warp head (a batch bound by its slowest points) the extra resident
    // warps slowed the head (768-speed sweep: 119 -> 136 ms).
    if (!trials && !any_head && b.shape.fp64 && !b.shape.nl && !b.shape.grouped &&
        b.shape.coop == 0) {
      KernelShape dk = b.shape;
      dk.dense = 1;
      int dbps = 0;
      if (occupancy_solve(dk, b.smem, &dbps) == 0 && 0.87 * dbps > (double)bps) {
        b.shape = dk;
        bps = dbps;
      }
    }
    b.blocks_per_sm = bps;
    b.grid = (int)std::min<long long>(b.count, (long long)bps * ctx->sms);
    buckets.push_back(b);
    return MCS_OK;
  };
  int rc = MCS_OK;
  std::vector<char> in_head(n_all, 0);
  any_head = !trials && pp && coop_warps > 1 && coop_head > 0;
  if (any_head) {
    std::vector<int32_t> members;
    std::vector<Bucket> heads;
    coop_head_buckets(cost, slots, modes, nls, grps, *pp, fp64, coop_warps, coop_head,
                      members, heads);
    order.insert(order.end(), members.begin(), members.end());
    for (int32_t q : members) in_head[q] = 1;
    for (Bucket& b : heads)
      if ((rc = place(b))) return rc;
    nbmax = std::min(nbmax, kMaxBuckets - (int)heads.size());
  }
  int classes = 0;
  std::vector<int32_t> idx;
  idx.reserve(n_all);
  for (size_t q = 0; q < n_all; q++)
    if (!in_head[q]) idx.push_back((int32_t)q);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return smem[a] > smem[b]; });
  const size_t n = idx.size();
  const double hi = n ? smem[idx.front()] : 1.0, lo = n ? std::max(1, smem[idx.back()]) : 1.0;
  // size classes: a bucket holds the points within a factor `ratio` of its largest need
  const double ratio = std::max(1.1, std::pow(hi / lo, 1.0 / nbmax) * 1.0001);
  size_t i = 0;
  while (i < n) {
    Bucket b;
    const int top = smem[idx[i]];
    size_t j = i;
    int sl = 1, nm = 1, nl = 0, gr = 0;
    while (j < n && (double)smem[idx[j]] * ratio >= top) {
      sl = std::max(sl, slots[idx[j]]);
      nm = std::max(nm, modes[idx[j]]);
      nl = std::max(nl, nls[idx[j]]);
      gr = std::max(gr, grps[idx[j]]);
      j++;
    }
    if (++classes == nbmax) {  // last bucket takes the rest
      for (size_t k = j; k < n; k++) {
        sl = std::max(sl, slots[idx[k]]);
        nm = std::max(nm, modes[idx[k]]);
        nl = std::max(nl, nls[idx[k]]);
        gr = std::max(gr, grps[idx[k]]);
      }
      j = n;
    }
    std::vector<int32_t> seg(idx.begin() + i, idx.begin() + j);
    std::stable_sort(seg.begin(), seg.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    b.offset = (int)order.size();
    b.count = (int)seg.size();
    b.smem = (top + 15) & ~15;
    b.shape = KernelShape{sl, nm, fp64, nl, trials ? 0 : gr};
    order.insert(order.end(), seg.begin(), seg.end());
    if ((rc = place(b))) return rc;
    i = j;
  }
  return MCS_OK;
}

DevOpts dev_opts(const mcs_opts* o) {
  DevOpts d;
  d.a_min = o->a_min;
  d.a_max = o->a_max;
  d.chatter_idx = o->chatter_idx;
  d.iters = o->iters;
  d.pad = 0;
  return d;
}

// The surrogate's predictions for a guided plan's points (features already on the device).
int enqueue_guide(mcs_plan* pl, cudaStream_t s0) {
  if (!pl->sur || pl->n == 0) return MCS_OK;
  return surrogate_predict_device(pl->sur, static_cast<const float*>(pl->feat.p), (long)pl->n,
                                  static_cast<float*>(pl->gmu.p),
                                  static_cast<float*>(pl->gsigma.p),
                                  static_cast<float2*>(pl->guide.p), &pl->gopts, s0,
                                  pl->a_max);
}

// Enqueue the plan's work: zero the queue counters, (optionally) the surrogate's
// predictions, then the buckets, longest points first.
//  - Captured (a plan's graph): one chain of programmatic dependent launches on the same
//    stream.  Each bucket's kernel starts once every block of the one before is resident,
//    so the long points always take the SMs first.  Parallel graph branches, one per
//    bucket, start in an unspecified order: the sweep ran 204 or 243 ms from one
//    execution to the next.
//  - Direct calls: one stream per bucket, forked and joined; the launches reach the device
//    in issue order.  A chain of more than 8 dependent launches outside a graph ran the
//    sweep in 309 ms instead of 199 ms.
// Captured plans leave the predictions out of the graph and run them just before it
// (mcs_plan_execute): with the inference kernel inside the graph the same bucket kernels
// ran 7 % slower on 65536 serving queries.
int enqueue(mcs_plan* pl, cudaStream_t s0, const mcs_opts* o, const volatile int* cancel,
            unsigned int* progress, double chatter_idx, bool with_guide = true,
            bool captured = false) {
  mcs_ctx* ctx = pl->ctx;
  const int nb = (int)pl->buckets.size();
  MCS_CUDA(cudaMemsetAsync(pl->queues.p, 0, sizeof(unsigned int) * std::max(1, nb), s0));
  if (progress) MCS_CUDA(cudaMemsetAsync(progress, 0, sizeof(unsigned int), s0));
  if (nb == 0) return MCS_OK;
  GuideArgs ga;
  if (pl->sur) {
    if (with_guide) {
      const int rc = enqueue_guide(pl, s0);
      if (rc) return rc;
    }
    ga.guide = static_cast<const float2*>(pl->guide.p);
    ga.sigma = static_cast<const float*>(pl->gsigma.p);
    ga.info = static_cast<mcs_guide_info*>(pl->ginfo.p);
    ga.hw_min = pl->gopts.hw_min;
    ga.refine = pl->gopts.refine;
    ga.mode = pl->gopts.mode;
    ga.levels = pl->gopts.levels;
  }
  const bool forked = !captured && nb > 1;
  if (forked) MCS_CUDA(cudaEventRecord(ctx->fork, s0));
  for (int b = 0; b < nb; b++) {
    const Bucket& bk = pl->buckets[b];
    // the first bucket waits for the memsets and the predictions like any stream work
    const bool chained = captured && b > 0;
    cudaStream_t sb = forked ? ctx->aux[b] : s0;
    if (forked) MCS_CUDA(cudaStreamWaitEvent(sb, ctx->fork, 0));
    unsigned int* q = static_cast<unsigned int*>(pl->queues.p) + b;
    const int32_t* order = static_cast<const int32_t*>(pl->order.p) + bk.offset;
    int rc;
    // buckets come in decreasing shared-memory need, i.e. longest points first; they also
    // get decreasing block priorities for the SMs that free up while several run
    const int prio = std::min(ctx->prio_low, ctx->prio_high + b);
    if (pl->trials)
      rc = launch_trials(bk.shape, bk.grid, bk.smem, sb,
                         static_cast<const PointParams*>(pl->params.p),
                         static_cast<const TrialItem*>(pl->items.p) + bk.offset, bk.count,
                         chatter_idx, static_cast<mcs_trial_result*>(pl->results.p), q, prio,
                         chained);
    else
      rc = launch_solve(bk.shape, bk.grid, bk.smem, sb,
                        static_cast<const PointParams*>(pl->params.p), order, bk.count,
                        dev_opts(o), static_cast<mcs_result*>(pl->results.p), q, cancel,
                        progress, ga, prio, chained);
    if (rc != 0)
      return fail(MCS_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString((cudaError_t)rc));
    if (forked) {
      MCS_CUDA(cudaEventRecord(ctx->join[b], sb));
      MCS_CUDA(cudaStreamWaitEvent(s0, ctx->join[b], 0));
    }
  }
  return MCS_OK;
}

void plan_free(mcs_plan* pl) {
  if (!pl) return;
  if (pl->exec) cudaGraphExecDestroy(pl->exec);
  if (pl->graph) cudaGraphDestroy(pl->graph);
  pl->params.release();
  pl->order.release();
  pl->results.release();
  pl->queues.release();
  pl->items.release();
  pl->feat.release();
  pl->gmu.release();
  pl->gsigma.release();
  pl->guide.release();
  pl->ginfo.release();
  if (pl->sur) surrogate_hold(pl->sur, -1);
  delete pl;
}

// Copies two host arrays to the device through the context's page-locked staging buffer
// and waits for the copies (the staging buffer is reused by the next call).
int upload2(mcs_ctx* ctx, cudaStream_t stream, void* d1, const void* h1, size_t n1, void* d2,
            const void* h2, size_t n2) {
  const size_t off2 = (n1 + 255) & ~size_t(255);
  const size_t need = off2 + n2;
  if (need > ctx->pinned_cap) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_cap = 0;
    const size_t want = std::max<size_t>(need, 1 << 20);
    cudaError_t e = cudaHostAlloc(&ctx->pinned, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      ctx->pinned = nullptr;
      return fail(MCS_ERR_NOMEM, "cudaHostAlloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    ctx->pinned_cap = want;
  }
  char* st = static_cast<char*>(ctx->pinned);
  std::memcpy(st, h1, n1);
  if (n2) std::memcpy(st + off2, h2, n2);
  MCS_CUDA(cudaMemcpyAsync(d1, st, n1, cudaMemcpyHostToDevice, stream));
  if (n2) MCS_CUDA(cudaMemcpyAsync(d2, st + off2, n2, cudaMemcpyHostToDevice, stream));
  MCS_CUDA(cudaStreamSynchronize(stream));
  return MCS_OK;
}

// Validates, prepares and uploads a solve batch; optionally captures it in a graph.
int build_plan(mcs_ctx* ctx, const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
               size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* o,
               bool capture, cudaStream_t stream, mcs_plan** out,
               mcs_surrogate* sur = nullptr, const mcs_guide_opts* g = nullptr,
               mcs_plan* reuse = nullptr) {
  int rc = check_inputs(setups, n_setups, modals, n_modals, points, n_points, o);
  if (rc) return rc;
  if (sur && (!g || !(g->z > 0) || !(g->hw_min > 0) || !(g->hw_max >= g->hw_min) ||
              !(g->hw_direct > 0) || g->refine < 0 || g->refine > 30 ||
              (g->mode != MCS_GUIDE_SPECULATE && g->mode != MCS_GUIDE_BRACKET) ||
              (g->mode == MCS_GUIDE_SPECULATE && g->levels < 1) ||
              !(g->skip_top >= 0.f && g->skip_top <= 1.f)))
    return fail(MCS_ERR_ARG, "guide options out of range");
  std::vector<PointParams> pp(n_points);
  std::vector<int> smem(n_points), slots(n_points), modes(n_points), nls(n_points),
      grps(n_points);
  std::vector<double> cost(n_points);
  for (size_t i = 0; i < n_points; i++) {
    Prepared pr;
    rc = prepare_point(setups[points[i].setup], modals[points[i].modal], points[i].S, *o,
                       o->a_max, pr);
    if (rc) return fail(rc, "point %zu: %s", i, g_last_error.c_str());
    pp[i] = pr.pp;
    smem[i] = pr.pp.smem_bytes;
    slots[i] = slots_for(pr.pp.nz_max);
    modes[i] = pr.modes;
    nls[i] = pr.nl;
    grps[i] = pr.pp.groups > 1 ? 1 : 0;
    cost[i] = pr.cost;
  }
  // a reused plan keeps its device buffers (they only grow) and drops everything else
  mcs_plan* pl = reuse ? reuse : new mcs_plan();
  if (reuse) {
    pl->n = 0;
    pl->trials = false;
    pl->sur = nullptr;
    pl->buckets.clear();
    pl->max_modes = pl->max_slots = 1;
    pl->executed = false;
  }
  auto discard = [&](mcs_plan* q) {
    if (q != reuse) {
      plan_free(q);
    } else if (q->sur) {  // a reused plan keeps its buffers but not the surrogate
      surrogate_hold(q->sur, -1);
      q->sur = nullptr;
    }
  };
  pl->ctx = ctx;
  pl->n = n_points;
  std::vector<int32_t> order;
  // multi-warp bisection for plain solves.  The library's rule (both options 0) gives it to
  // the points whose serial bisections would outlast the rest of the batch (coop_auto_head);
  // a batch bound by its total work gets none, since the speculative trials add to it.
  int coop = 1, head = 0;
  if (!sur) {
    if (o->coop_warps == 0 && o->coop_points == 0) {
      head = coop_auto_head(ctx, smem, cost, slots, modes, nls, grps, o->precision == MCS_FP64);
      if (head > 0) coop = kCoopMaxWarpsHost;
    } else if (o->coop_warps != 1) {
      coop = o->coop_warps == 0 ? kCoopMaxWarpsHost : o->coop_warps;
      head = o->coop_points == 0 ? ctx->sms : o->coop_points;
    }
  }
  rc = make_buckets(ctx, smem, cost, slots, modes, nls, grps, false, o->precision == MCS_FP64,
                    o->max_buckets, order,
                    pl->buckets, &pp, coop, head);
  if (rc) {
    discard(pl);
    return rc;
  }
  const size_t nb = std::max<size_t>(1, pl->buckets.size());
  if ((rc = pl->params.ensure(sizeof(PointParams) * std::max<size_t>(1, n_points))) ||
      (rc = pl->order.ensure(sizeof(int32_t) * std::max<size_t>(1, n_points))) ||
      (rc = pl->results.ensure(sizeof(mcs_result) * std::max<size_t>(1, n_points))) ||
      (rc = pl->queues.ensure(sizeof(unsigned int) * nb))) {
    discard(pl);
    return rc;
  }
  if (n_points) {
    rc = upload2(ctx, stream, pl->params.p, pp.data(), sizeof(PointParams) * n_points,
                 pl->order.p, order.data(), sizeof(int32_t) * n_points);
    if (rc) {
      discard(pl);
      return rc;
    }
  }
  for (const Bucket& b : pl->buckets) {
    pl->max_modes = std::max(pl->max_modes, b.shape.modes);
    pl->max_slots = std::max(pl->max_slots, b.shape.slots);
  }
  if (sur && n_points) {
    pl->sur = sur;
    surrogate_hold(sur, +1);
    pl->gopts = *g;
    pl->a_max = o->a_max;
    std::vector<float> f(n_points * MCS_FEATURES);
    for (size_t i = 0; i < n_points; i++)
      point_features(setups[points[i].setup], modals[points[i].modal], points[i].S, *o,
                     &f[i * MCS_FEATURES]);
    if ((rc = pl->feat.ensure(sizeof(float) * f.size())) ||
        (rc = pl->gmu.ensure(sizeof(float) * n_points)) ||
        (rc = pl->gsigma.ensure(sizeof(float) * n_points)) ||
        (rc = pl->guide.ensure(sizeof(float2) * n_points)) ||
        (rc = pl->ginfo.ensure(sizeof(mcs_guide_info) * n_points)) ||
        (rc = surrogate_reserve(sur))) {
      discard(pl);
      return rc;
    }
    cudaError_t e = cudaMemcpyAsync(pl->feat.p, f.data(), sizeof(float) * f.size(),
                                    cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      discard(pl);
      return fail(MCS_ERR_CUDA, "feature upload failed: %s", cudaGetErrorString(e));
    }
  }
  if (capture) {
    cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      discard(pl);
      return fail(MCS_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    }
    rc = enqueue(pl, stream, o, nullptr, nullptr, o->chatter_idx, /*with_guide=*/false,
                 /*captured=*/true);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(stream, &g);
    if (rc || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      discard(pl);
      return rc ? rc : fail(MCS_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    }
    pl->graph = g;
    e = cudaGraphInstantiate(&pl->exec, g, 0);
    if (e != cudaSuccess) {
      discard(pl);
      return fail(MCS_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    }
  }
  *out = pl;
  return MCS_OK;
}

}  // namespace

extern "C" {

void mcs_default_opts(mcs_opts* o) {
  if (!o) return;
  o->a_min = 0.05;
  o->a_max = 20.0;
  o->iters = 8;
  o->revs = 120;
  o->nonlinear = 1;
  o->honor_runout = 0;
  o->steps_per_tooth = 0;
  o->slices = 0;
  o->chatter_idx = 0.45;
  o->precision = MCS_FP64;  // the reference's arithmetic; MCS_FP32 is the faster variant
  o->max_buckets = 0;
  o->serial_trials = 0;
  o->coop_warps = 0;
  o->coop_points = 0;
  o->pad = 0;
}

const char* mcs_last_error(void) { return g_last_error.c_str(); }

int mcs_create(mcs_ctx** out, int device) {
  if (!out) return fail(MCS_ERR_ARG, "ctx pointer is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(MCS_ERR_CUDA, "no CUDA device: %s",
                e != cudaSuccess ? cudaGetErrorString(e) : "device count is 0");
  if (device < 0 || device >= count)
    return fail(MCS_ERR_ARG, "device %d out of range (%d devices)", device, count);
  MCS_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  MCS_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(MCS_ERR_UNSUPPORTED, "device %d is sm_%d%d; the kernels are built for sm_100a",
                device, prop.major, prop.minor);
  const int rc = set_smem_limits();
  if (rc) return fail(MCS_ERR_CUDA, "kernel attributes: %s", cudaGetErrorString((cudaError_t)rc));
  mcs_ctx* c = new mcs_ctx();
  c->device = device;
  c->sms = prop.multiProcessorCount;
  MCS_CUDA(cudaDeviceGetStreamPriorityRange(&c->prio_low, &c->prio_high));
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int b = 0; ok && b < kMaxBuckets; b++)
    ok = cudaStreamCreateWithFlags(&c->aux[b], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&c->join[b], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    mcs_destroy(c);
    return fail(MCS_ERR_CUDA, "stream/event creation failed");
  }
  *out = c;
  return MCS_OK;
}

int mcs_destroy(mcs_ctx* c) {
  if (!c) return MCS_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  plan_free(c->solve_scratch);
  plan_free(c->guided_scratch);
  for (int b = 0; b < kMaxBuckets; b++) {
    if (c->aux[b]) cudaStreamDestroy(c->aux[b]);
    if (c->join[b]) cudaEventDestroy(c->join[b]);
  }
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->pinned) cudaFreeHost(c->pinned);
  delete c;
  return MCS_OK;
}

void* mcs_stream(mcs_ctx* c) { return c ? (void*)c->stream : nullptr; }

int mcs_plan_create(mcs_ctx* c, const mcs_setup* setups, size_t n_setups,
                    const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                    size_t n_points, const mcs_opts* opts, mcs_plan** plan) {
  if (!c || !plan) return fail(MCS_ERR_ARG, "NULL ctx or plan pointer");
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  return build_plan(c, setups, n_setups, modals, n_modals, points, n_points, opts, true,
                    c->stream, plan);
}

int mcs_plan_execute(mcs_plan* pl) {
  if (!pl) return fail(MCS_ERR_ARG, "plan is NULL");
  std::lock_guard<std::mutex> lk(pl->ctx->mu);
  MCS_CUDA(cudaSetDevice(pl->ctx->device));
  if (pl->exec) {
    const int rc = enqueue_guide(pl, pl->ctx->stream);
    if (rc) return rc;
    MCS_CUDA(cudaGraphLaunch(pl->exec, pl->ctx->stream));
  }
  pl->executed = true;
  return MCS_OK;
}

int mcs_plan_results(mcs_plan* pl, mcs_result* out) {
  if (!pl || (!out && pl->n)) return fail(MCS_ERR_ARG, "NULL plan or output");
  if (!pl->executed) return fail(MCS_ERR_STATE, "plan was never executed");
  std::lock_guard<std::mutex> lk(pl->ctx->mu);
  MCS_CUDA(cudaSetDevice(pl->ctx->device));
  if (pl->n)
    MCS_CUDA(cudaMemcpyAsync(out, pl->results.p, sizeof(mcs_result) * pl->n,
                             cudaMemcpyDeviceToHost, pl->ctx->stream));
  MCS_CUDA(cudaStreamSynchronize(pl->ctx->stream));
  return pl->sur ? surrogate_check(pl->sur) : MCS_OK;
}

int mcs_plan_info_get(const mcs_plan* pl, mcs_plan_info* info) {
  if (!pl || !info) return fail(MCS_ERR_ARG, "NULL plan or info");
  std::memset(info, 0, sizeof(*info));
  int warps = 0, smem = 0;
  for (const Bucket& b : pl->buckets) {
    info->blocks += b.grid;
    warps = std::max(warps, b.blocks_per_sm * std::max(1, b.shape.coop));
    smem = std::max(smem, b.smem);
    if (b.shape.coop > 0) info->coop_points += b.count;
  }
  info->warps_per_sm = warps;
  info->smem_per_warp = smem;
  info->slots = pl->max_slots;
  info->modes = pl->max_modes;
  info->graph = pl->exec ? 1 : 0;
  info->kernels = (int)pl->buckets.size() + (pl->sur ? 1 : 0);  // + the inference kernel
  info->n_points = pl->n;
  info->h2d_bytes = pl->trials ? 0 : (uint64_t)pl->n * (sizeof(PointParams) + sizeof(int32_t));
  info->d2h_bytes = pl->trials ? 0 : (uint64_t)pl->n * sizeof(mcs_result);
  return MCS_OK;
}

int mcs_plan_destroy(mcs_plan* pl) {
  if (!pl) return MCS_OK;
  {
    std::lock_guard<std::mutex> lk(pl->ctx->mu);
    cudaSetDevice(pl->ctx->device);
    cudaStreamSynchronize(pl->ctx->stream);
  }
  plan_free(pl);
  return MCS_OK;
}

int mcs_tune(mcs_ctx* c, const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
             size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* opts,
             const int32_t* candidates, size_t n_candidates, double* ms, int32_t* best) {
  if (!c || !opts || !best) return fail(MCS_ERR_ARG, "NULL ctx, opts or best");
  if (n_candidates == 0 || !candidates) return fail(MCS_ERR_ARG, "no candidate schedules");
  if (n_candidates > 64) return fail(MCS_ERR_ARG, "at most 64 candidate schedules");
  for (size_t i = 0; i < n_candidates; i++)
    if (candidates[i] < 1 || candidates[i] > kMaxBuckets)
      return fail(MCS_ERR_ARG, "candidate %zu: max_buckets %d out of range [1, %d]", i,
                  candidates[i], kMaxBuckets);
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  // all candidate plans first; then kRounds rounds in which every candidate runs once,
  // round-robin, so that a drift of the clocks does not favour one candidate; each
  // candidate's time is its mean over the rounds: schedules with many concurrent grids
  // vary from run to run (their start order races), and a best-of ranking chose them
  constexpr int kRounds = 3;
  std::vector<mcs_plan*> plans(n_candidates, nullptr);
  std::vector<double> t(n_candidates, 0.0);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = MCS_OK;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    rc = fail(MCS_ERR_CUDA, "event creation failed");
  // every timed run starts from a cold L2, as after unrelated work: a schedule measured
  // back to back on a warm L2 ranked differently (24 classes: 200 ms warm, 250-300 ms cold)
  int l2 = 0;
  cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device);
  const size_t flush_bytes = 2 * (size_t)std::max(l2, 1 << 20);
  void* flush = nullptr;
  if (!rc && cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
    flush = nullptr;
    rc = fail(MCS_ERR_NOMEM, "no room for the L2 flush buffer (%zu bytes)", flush_bytes);
  }
  for (size_t i = 0; i < n_candidates && !rc; i++) {
    mcs_opts o = *opts;
    o.max_buckets = candidates[i];
    rc = build_plan(c, setups, n_setups, modals, n_modals, points, n_points, &o, true, c->stream,
                    &plans[i]);
  }
  cudaError_t e = cudaSuccess;
  for (int r = -1; r < kRounds && !rc && e == cudaSuccess; r++) {
    for (size_t i = 0; i < n_candidates && e == cudaSuccess; i++) {
      if (!plans[i]->exec) {
        t[i] = 0.0;
        continue;
      }
      if (r < 0) {  // untimed: the first launch uploads the graph
        e = cudaGraphLaunch(plans[i]->exec, c->stream);
        continue;
      }
      float f = 0.f;
      e = cudaMemsetAsync(flush, (r * 31 + (int)i) & 0xFF, flush_bytes, c->stream);
      if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
      if (e == cudaSuccess) e = cudaGraphLaunch(plans[i]->exec, c->stream);
      if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
      if (e == cudaSuccess) t[i] += (double)f / kRounds;
    }
  }
  cudaStreamSynchronize(c->stream);
  for (mcs_plan* pl : plans) plan_free(pl);
  if (flush) cudaFree(flush);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!rc && e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "tuning run failed: %s", cudaGetErrorString(e));
  if (rc) return rc;
  size_t bi = 0;
  for (size_t i = 0; i < n_candidates; i++) {
    if (ms) ms[i] = t[i];
    if (t[i] < t[bi]) bi = i;
  }
  *best = candidates[bi];
  return MCS_OK;
}

int mcs_solve(mcs_ctx* c, const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
              size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* opts,
              mcs_result* out) {
  if (!c) return fail(MCS_ERR_ARG, "ctx is NULL");
  if (n_points && !out) return fail(MCS_ERR_ARG, "out is NULL");
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  mcs_plan* pl = nullptr;
  // the context's solve plan is reused: its device buffers persist between calls, so a
  // repeated solve of a similar batch neither allocates nor frees device memory
  if (!c->solve_scratch) c->solve_scratch = new mcs_plan();
  int rc = build_plan(c, setups, n_setups, modals, n_modals, points, n_points, opts, false,
                      c->stream, &pl, nullptr, nullptr, c->solve_scratch);
  if (rc) return rc;
  rc = enqueue(pl, c->stream, opts, nullptr, nullptr, opts->chatter_idx);
  if (!rc && n_points) {
    cudaError_t e = cudaMemcpyAsync(out, pl->results.p, sizeof(mcs_result) * n_points,
                                    cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "result copy failed: %s", cudaGetErrorString(e));
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (!rc && e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "solve failed: %s", cudaGetErrorString(e));
  return rc;
}

int mcs_shard(const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
              size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* o,
              size_t n_shards, int32_t* shard_of, double* cost_out) {
  if (n_shards < 1 || n_shards > 4096) return fail(MCS_ERR_ARG, "n_shards out of range [1, 4096]");
  if (n_points && !shard_of) return fail(MCS_ERR_ARG, "shard_of is NULL");
  int rc = check_inputs(setups, n_setups, modals, n_modals, points, n_points, o);
  if (rc) return rc;
  std::vector<double> cost(n_points);
  for (size_t i = 0; i < n_points; i++) {
    Prepared pr;
    rc = prepare_point(setups[points[i].setup], modals[points[i].modal], points[i].S, *o,
                       o->a_max, pr);
    if (rc) return fail(rc, "point %zu: %s", i, g_last_error.c_str());
    cost[i] = pr.cost;
  }
  std::vector<size_t> order(n_points);
  std::iota(order.begin(), order.end(), size_t(0));
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return cost[a] > cost[b]; });
  // least-loaded shard first, the lower index among equal loads
  using Load = std::pair<double, size_t>;
  std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
  for (size_t k = 0; k < n_shards; k++) heap.push({0.0, k});
  for (size_t i : order) {
    const Load l = heap.top();
    heap.pop();
    shard_of[i] = (int32_t)l.second;
    heap.push({l.first + cost[i], l.second});
  }
  if (cost_out) std::copy(cost.begin(), cost.end(), cost_out);
  return MCS_OK;
}

int mcs_solve_multi(mcs_ctx* const* ctxs, size_t n_ctx, const mcs_setup* setups,
                    size_t n_setups, const mcs_modal* modals, size_t n_modals,
                    const mcs_point* points, size_t n_points, const mcs_opts* o,
                    mcs_result* out) {
  if (!ctxs || n_ctx == 0) return fail(MCS_ERR_ARG, "no contexts");
  for (size_t k = 0; k < n_ctx; k++)
    if (!ctxs[k]) return fail(MCS_ERR_ARG, "context %zu is NULL", k);
  if (n_points && !out) return fail(MCS_ERR_ARG, "out is NULL");
  std::vector<int32_t> shard_of(n_points);
  int rc = mcs_shard(setups, n_setups, modals, n_modals, points, n_points, o, n_ctx,
                     shard_of.data(), nullptr);
  if (rc) return rc;
  std::vector<std::vector<size_t>> idx(n_ctx);
  for (size_t i = 0; i < n_points; i++) idx[shard_of[i]].push_back(i);
  std::vector<int> status(n_ctx, MCS_OK);
  std::vector<std::string> message(n_ctx);
  std::vector<std::vector<mcs_result>> res(n_ctx);
  auto work = [&](size_t k) {
    std::vector<mcs_point> pts(idx[k].size());
    for (size_t j = 0; j < pts.size(); j++) pts[j] = points[idx[k][j]];
    res[k].resize(pts.size());
    status[k] = mcs_solve(ctxs[k], setups, n_setups, modals, n_modals, pts.data(), pts.size(), o,
                          res[k].data());
    if (status[k]) message[k] = g_last_error;  // this thread's message
  };
  std::vector<std::thread> pool;
  for (size_t k = 1; k < n_ctx; k++) pool.emplace_back(work, k);
  work(0);
  for (std::thread& t : pool) t.join();
  for (size_t k = 0; k < n_ctx; k++)
    if (status[k]) return fail(status[k], "shard %zu: %s", k, message[k].c_str());
  for (size_t k = 0; k < n_ctx; k++)
    for (size_t j = 0; j < idx[k].size(); j++) out[idx[k][j]] = res[k][j];
  return MCS_OK;
}

int mcs_chatter_at(mcs_ctx* c, const mcs_setup* setups, size_t n_setups,
                   const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                   size_t n_points, const mcs_trial* trials, size_t n_trials,
                   const mcs_opts* o, mcs_trial_result* out) {
  if (!c) return fail(MCS_ERR_ARG, "ctx is NULL");
  if (n_trials && (!trials || !out)) return fail(MCS_ERR_ARG, "NULL trials or output");
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  int rc = check_inputs(setups, n_setups, modals, n_modals, points, n_points, o);
  if (rc) return rc;
  if (n_trials > (size_t)std::numeric_limits<int32_t>::max())
    return fail(MCS_ERR_ARG, "too many trials");
  double ap_max = 0;
  for (size_t i = 0; i < n_trials; i++) {
    if (trials[i].point >= n_points)
      return fail(MCS_ERR_ARG, "trial %zu: point index out of range", i);
    if (!(is_finite(trials[i].ap) && trials[i].ap > 0 && trials[i].ap < 1e4))
      return fail(MCS_ERR_ARG, "trial %zu: ap must be in (0, 1e4)", i);
  }
  // per point: the deepest trial sets its slice count
  std::vector<double> deepest(n_points, 0.0);
  for (size_t i = 0; i < n_trials; i++)
    deepest[trials[i].point] = std::max(deepest[trials[i].point], trials[i].ap);
  std::vector<PointParams> pp(n_points);
  std::vector<int> modes(n_points), pnl(n_points);
  for (size_t i = 0; i < n_points; i++) {
    Prepared pr;
    ap_max = deepest[i] > 0 ? deepest[i] : o->a_min;
    rc = prepare_point(setups[points[i].setup], modals[points[i].modal], points[i].S, *o,
                       ap_max, pr);
    if (rc) return fail(rc, "point %zu: %s", i, g_last_error.c_str());
    pp[i] = pr.pp;
    modes[i] = pr.modes;
    pnl[i] = pr.nl;
  }
  std::vector<int> smem(n_trials), slots(n_trials), tmodes(n_trials), tnl(n_trials);
  std::vector<double> cost(n_trials);
  std::vector<TrialItem> items_by_idx(n_trials);
  for (size_t i = 0; i < n_trials; i++) {
    const PointParams& P = pp[trials[i].point];
    const int nz = slices_at(trials[i].ap, P.flute_len, o->slices);
    smem[i] = warp_smem(P.spr, o->precision == MCS_FP64, nz, P.lpad, 1);
    slots[i] = slots_for(nz);
    tmodes[i] = modes[trials[i].point];
    tnl[i] = pnl[trials[i].point];
    cost[i] = (double)P.nsteps * (24.0 + 40.0 * P.N * slots[i]);
    items_by_idx[i] = TrialItem{(int32_t)trials[i].point, (int32_t)i, trials[i].ap};
  }
  mcs_plan* pl = new mcs_plan();
  pl->ctx = c;
  pl->trials = true;
  pl->n = n_trials;
  std::vector<int32_t> order;
  rc = make_buckets(c, smem, cost, slots, tmodes, tnl, std::vector<int>(n_trials, 0), true,
                    o->precision == MCS_FP64,
                    o->max_buckets, order,
                    pl->buckets);
  std::vector<TrialItem> items(n_trials);
  for (size_t k = 0; k < order.size(); k++) items[k] = items_by_idx[order[k]];
  const size_t nb = std::max<size_t>(1, pl->buckets.size());
  if (!rc) rc = pl->params.ensure(sizeof(PointParams) * std::max<size_t>(1, n_points));
  if (!rc) rc = pl->items.ensure(sizeof(TrialItem) * std::max<size_t>(1, n_trials));
  if (!rc) rc = pl->results.ensure(sizeof(mcs_trial_result) * std::max<size_t>(1, n_trials));
  if (!rc) rc = pl->queues.ensure(sizeof(unsigned int) * nb);
  if (!rc) rc = pl->order.ensure(sizeof(int32_t));
  cudaError_t e = cudaSuccess;
  if (!rc && n_trials)
    rc = upload2(c, c->stream, pl->params.p, pp.data(), sizeof(PointParams) * n_points,
                 pl->items.p, items.data(), sizeof(TrialItem) * n_trials);
  if (!rc) rc = enqueue(pl, c->stream, o, nullptr, nullptr, o->chatter_idx);
  if (!rc && n_trials) {
    e = cudaMemcpyAsync(out, pl->results.p, sizeof(mcs_trial_result) * n_trials,
                        cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "result copy failed: %s", cudaGetErrorString(e));
  }
  e = cudaStreamSynchronize(c->stream);
  if (!rc && e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "trials failed: %s", cudaGetErrorString(e));
  plan_free(pl);
  return rc;
}

int mcs_solve_async(mcs_ctx* c, const mcs_setup* setups, size_t n_setups,
                    const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                    size_t n_points, const mcs_opts* opts, mcs_result* out, mcs_job** job) {
  if (!c || !job) return fail(MCS_ERR_ARG, "NULL ctx or job pointer");
  if (n_points && !out) return fail(MCS_ERR_ARG, "out is NULL");
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  *job = nullptr;
  mcs_job* jb = new mcs_job();
  jb->out = out;
  auto bail = [&](int code) {
    if (jb->plan) plan_free(jb->plan);
    jb->cancel.release();
    jb->progress.release();
    if (jb->staging) cudaFreeHost(jb->staging);
    if (jb->done) cudaEventDestroy(jb->done);
    if (jb->stream) cudaStreamDestroy(jb->stream);
    delete jb;
    return code;
  };
  if (cudaStreamCreateWithFlags(&jb->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&jb->done, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(MCS_ERR_CUDA, "job stream/event creation failed"));
  int rc = build_plan(c, setups, n_setups, modals, n_modals, points, n_points, opts, false,
                      jb->stream, &jb->plan);
  if (rc) return bail(rc);
  if ((rc = jb->cancel.ensure(sizeof(int))) || (rc = jb->progress.ensure(sizeof(unsigned int))))
    return bail(rc);
  if (cudaHostAlloc((void**)&jb->staging, sizeof(mcs_result) * std::max<size_t>(1, n_points),
                    cudaHostAllocDefault) != cudaSuccess)
    return bail(fail(MCS_ERR_NOMEM, "pinned staging allocation failed"));
  if (cudaMemsetAsync(jb->cancel.p, 0, sizeof(int), jb->stream) != cudaSuccess)
    return bail(fail(MCS_ERR_CUDA, "memset failed"));
  rc = enqueue(jb->plan, jb->stream, opts, static_cast<const volatile int*>(jb->cancel.p),
               static_cast<unsigned int*>(jb->progress.p), opts->chatter_idx);
  if (rc) return bail(rc);
  if (n_points &&
      cudaMemcpyAsync(jb->staging, jb->plan->results.p, sizeof(mcs_result) * n_points,
                      cudaMemcpyDeviceToHost, jb->stream) != cudaSuccess)
    return bail(fail(MCS_ERR_CUDA, "result copy failed"));
  if (cudaEventRecord(jb->done, jb->stream) != cudaSuccess)
    return bail(fail(MCS_ERR_CUDA, "event record failed"));
  *job = jb;
  return MCS_OK;
}

int mcs_job_poll(mcs_job* jb, size_t* points_done, int* finished) {
  if (!jb) return fail(MCS_ERR_ARG, "job is NULL");
  mcs_ctx* c = jb->plan->ctx;
  MCS_CUDA(cudaSetDevice(c->device));
  const cudaError_t q = cudaEventQuery(jb->done);
  if (q != cudaSuccess && q != cudaErrorNotReady)
    return fail(MCS_ERR_CUDA, "job failed: %s", cudaGetErrorString(q));
  if (finished) *finished = q == cudaSuccess ? 1 : 0;
  if (points_done) {
    if (q == cudaSuccess) {
      *points_done = jb->plan->n;
    } else {
      unsigned int v = 0;
      MCS_CUDA(cudaMemcpyAsync(&v, jb->progress.p, sizeof(v), cudaMemcpyDeviceToHost, c->side));
      MCS_CUDA(cudaStreamSynchronize(c->side));
      *points_done = v;
    }
  }
  return MCS_OK;
}

int mcs_job_cancel(mcs_job* jb) {
  if (!jb) return fail(MCS_ERR_ARG, "job is NULL");
  mcs_ctx* c = jb->plan->ctx;
  MCS_CUDA(cudaSetDevice(c->device));
  static const int one = 1;
  MCS_CUDA(cudaMemcpyAsync(jb->cancel.p, &one, sizeof(int), cudaMemcpyHostToDevice, c->side));
  MCS_CUDA(cudaStreamSynchronize(c->side));
  return MCS_OK;
}

int mcs_job_wait(mcs_job* jb) {
  if (!jb) return fail(MCS_ERR_ARG, "job is NULL");
  MCS_CUDA(cudaSetDevice(jb->plan->ctx->device));
  MCS_CUDA(cudaEventSynchronize(jb->done));
  if (!jb->waited && jb->plan->n) std::memcpy(jb->out, jb->staging, sizeof(mcs_result) * jb->plan->n);
  jb->waited = true;
  for (size_t i = 0; i < jb->plan->n; i++)
    if (jb->out[i].status == MCS_ERR_CANCELLED)
      return fail(MCS_ERR_CANCELLED, "job was cancelled; %zu points have results", i);
  return MCS_OK;
}

void mcs_job_free(mcs_job* jb) {
  if (!jb) return;
  cudaSetDevice(jb->plan->ctx->device);
  cudaEventSynchronize(jb->done);
  plan_free(jb->plan);
  jb->cancel.release();
  jb->progress.release();
  if (jb->staging) cudaFreeHost(jb->staging);
  cudaEventDestroy(jb->done);
  cudaStreamDestroy(jb->stream);
  delete jb;
}

int mcs_features(const mcs_setup* setups, size_t n_setups, const mcs_modal* modals,
                 size_t n_modals, const mcs_point* points, size_t n_points, const mcs_opts* o,
                 float* out) {
  if (n_points && !out) return fail(MCS_ERR_ARG, "out is NULL");
  int rc = check_inputs(setups, n_setups, modals, n_modals, points, n_points, o);
  if (rc) return rc;
  for (size_t i = 0; i < n_points; i++)
    point_features(setups[points[i].setup], modals[points[i].modal], points[i].S, *o,
                   out + i * MCS_FEATURES);
  return MCS_OK;
}

int mcs_solve_guided(mcs_ctx* c, mcs_surrogate* sur, const mcs_setup* setups, size_t n_setups,
                     const mcs_modal* modals, size_t n_modals, const mcs_point* points,
                     size_t n_points, const mcs_opts* opts, const mcs_guide_opts* g,
                     mcs_result* out, mcs_guide_info* info) {
  if (!c || !sur) return fail(MCS_ERR_ARG, "NULL ctx or surrogate");
  if (surrogate_ctx(sur) != c) return fail(MCS_ERR_ARG, "surrogate belongs to another context");
  if (n_points && !out) return fail(MCS_ERR_ARG, "out is NULL");
  std::lock_guard<std::mutex> lk(c->mu);
  std::lock_guard<std::mutex> slk(surrogate_mutex(sur));
  MCS_CUDA(cudaSetDevice(c->device));
  // the context's guided plan is reused like mcs_solve's: no device allocation per call
  if (!c->guided_scratch) c->guided_scratch = new mcs_plan();
  mcs_plan* pl = nullptr;
  int rc = build_plan(c, setups, n_setups, modals, n_modals, points, n_points, opts, false,
                      c->stream, &pl, sur, g, c->guided_scratch);
  if (rc) return rc;
  rc = enqueue(pl, c->stream, opts, nullptr, nullptr, opts->chatter_idx);
  if (!rc && n_points) {
    cudaError_t e = cudaMemcpyAsync(out, pl->results.p, sizeof(mcs_result) * n_points,
                                    cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && info)
      e = cudaMemcpyAsync(info, pl->ginfo.p, sizeof(mcs_guide_info) * n_points,
                          cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "result copy failed: %s", cudaGetErrorString(e));
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (!rc && e != cudaSuccess) rc = fail(MCS_ERR_CUDA, "guided solve failed: %s", cudaGetErrorString(e));
  if (!rc) rc = surrogate_check(sur);
  if (pl->sur) {  // the plan is kept for the next call; the surrogate is not held by it
    surrogate_hold(pl->sur, -1);
    pl->sur = nullptr;
  }
  return rc;
}

int mcs_plan_create_guided(mcs_ctx* c, mcs_surrogate* sur, const mcs_setup* setups,
                           size_t n_setups, const mcs_modal* modals, size_t n_modals,
                           const mcs_point* points, size_t n_points, const mcs_opts* opts,
                           const mcs_guide_opts* g, mcs_plan** plan) {
  if (!c || !sur || !plan) return fail(MCS_ERR_ARG, "NULL ctx, surrogate or plan pointer");
  if (surrogate_ctx(sur) != c) return fail(MCS_ERR_ARG, "surrogate belongs to another context");
  std::lock_guard<std::mutex> lk(c->mu);
  std::lock_guard<std::mutex> slk(surrogate_mutex(sur));
  MCS_CUDA(cudaSetDevice(c->device));
  return build_plan(c, setups, n_setups, modals, n_modals, points, n_points, opts, true,
                    c->stream, plan, sur, g);
}

int mcs_plan_guide_info(mcs_plan* pl, mcs_guide_info* info) {
  if (!pl || (!info && pl->n)) return fail(MCS_ERR_ARG, "NULL plan or output");
  if (!pl->sur) return fail(MCS_ERR_STATE, "the plan is not guided");
  if (!pl->executed) return fail(MCS_ERR_STATE, "plan was never executed");
  std::lock_guard<std::mutex> lk(pl->ctx->mu);
  MCS_CUDA(cudaSetDevice(pl->ctx->device));
  if (pl->n)
    MCS_CUDA(cudaMemcpyAsync(info, pl->ginfo.p, sizeof(mcs_guide_info) * pl->n,
                             cudaMemcpyDeviceToHost, pl->ctx->stream));
  MCS_CUDA(cudaStreamSynchronize(pl->ctx->stream));
  return MCS_OK;
}

int mcs_lobes_alim(mcs_ctx* c, const mcs_modal* modals, size_t n_modals,
                   const mcs_lobe_query* queries, size_t n_queries, const double* rpm,
                   size_t n_rpm, double* alim) {
  if (!c) return fail(MCS_ERR_ARG, "ctx is NULL");
  if (n_queries && n_rpm && (!modals || !queries || !rpm || !alim))
    return fail(MCS_ERR_ARG, "NULL input or output array");
  if (n_queries > 65535 * 64 || n_rpm > (size_t)std::numeric_limits<int32_t>::max())
    return fail(MCS_ERR_ARG, "too many queries or speeds");
  int rc = MCS_OK;
  for (size_t i = 0; i < n_modals; i++) {
    const mcs_modal& md = modals[i];
    if (md.nx < 1 || md.nx > kMaxModes || md.ny < 0 || md.ny > kMaxModes)
      return fail(MCS_ERR_ARG, "modal %zu: 1 <= nx <= %d and 0 <= ny <= %d", i, kMaxModes,
                  kMaxModes);
    for (int a = 0; a < 2; a++) {
      const int cnt = a == 0 ? md.nx : md.ny;
      const mcs_mode* ms = a == 0 ? md.x : md.y;
      for (int j = 0; j < cnt; j++)
        if (!(is_finite(ms[j].k) && ms[j].k > 0 && is_finite(ms[j].fn) && ms[j].fn > 0 &&
              is_finite(ms[j].zeta) && ms[j].zeta >= 0))
          return fail(MCS_ERR_ARG, "modal %zu: mode %d needs k > 0, fn > 0, zeta >= 0", i, j);
    }
  }
  for (size_t i = 0; i < n_queries; i++) {
    const mcs_lobe_query& q = queries[i];
    if (q.N < 1 || q.lobes < 0 || q.lobes > 10000 || q.modal >= n_modals ||
        !(is_finite(q.Ktc) && q.Ktc != 0 && is_finite(q.Krc) && is_finite(q.phi_st) &&
          is_finite(q.phi_ex) && is_finite(q.rpm_min) && is_finite(q.rpm_max)))
      return fail(MCS_ERR_ARG, "lobe query %zu is invalid", i);
  }
  for (size_t r = 0; r < n_rpm; r++)
    if (!is_finite(rpm[r])) return fail(MCS_ERR_ARG, "rpm %zu is not finite", r);
  if (!n_queries || !n_rpm) return MCS_OK;
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  DevBuf dm, dq, dr, dout;
  if ((rc = dm.ensure(sizeof(mcs_modal) * n_modals)) || (rc = dq.ensure(sizeof(mcs_lobe_query) * n_queries)) ||
      (rc = dr.ensure(sizeof(double) * n_rpm)) || (rc = dout.ensure(sizeof(double) * n_queries * n_rpm))) {
    dm.release(); dq.release(); dr.release(); dout.release();
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(dm.p, modals, sizeof(mcs_modal) * n_modals, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dq.p, queries, sizeof(mcs_lobe_query) * n_queries, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dr.p, rpm, sizeof(double) * n_rpm, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = (cudaError_t)launch_lobes(c->stream, static_cast<const mcs_modal*>(dm.p),
                                  static_cast<const mcs_lobe_query*>(dq.p), (int)n_queries,
                                  static_cast<const double*>(dr.p), (int)n_rpm,
                                  static_cast<double*>(dout.p));
  if (e == cudaSuccess) e = cudaMemcpyAsync(alim, dout.p, sizeof(double) * n_queries * n_rpm, cudaMemcpyDeviceToHost, c->stream);
  cudaError_t e2 = cudaStreamSynchronize(c->stream);
  dm.release(); dq.release(); dr.release(); dout.release();
  if (e != cudaSuccess) return fail(MCS_ERR_CUDA, "lobes failed: %s", cudaGetErrorString(e));
  if (e2 != cudaSuccess) return fail(MCS_ERR_CUDA, "lobes failed: %s", cudaGetErrorString(e2));
  return MCS_OK;
}

int mcs_lobes_composite(mcs_ctx* c, const mcs_spindle* sp, const mcs_speed_frf* frfs,
                        size_t n_frfs, const mcs_lobe_query* base, double* rpm_out,
                        double* alim_out, size_t cap, size_t* n_out) {
  if (!c || !sp || !base || !n_out) return fail(MCS_ERR_ARG, "NULL ctx, spindle, base or n_out");
  const mcs_lobe_query& B = *base;
  if (B.N < 1 || B.lobes < 0 || B.lobes > 10000 ||
      !(is_finite(B.Ktc) && B.Ktc != 0 && is_finite(B.Krc) && is_finite(B.phi_st) &&
        is_finite(B.phi_ex) && is_finite(B.rpm_min) && is_finite(B.rpm_max)))
    return fail(MCS_ERR_ARG, "base lobe query is invalid");
  // the nodes and their speeds, as Simulator.lobes walks them (sim.js:275-281)
  const double lo = B.rpm_min * 0.8, hi = B.rpm_max * 1.1;
  if ((hi - lo) / MCS_LOBE_NODE > 100000)
    return fail(MCS_ERR_ARG, "speed range of %g rpm is too wide", hi - lo);
  std::vector<double> centre, samples;
  std::vector<mcs_lobe_query> qs;
  std::vector<int> begin, count;
  for (double S0 = lo; S0 < hi; S0 += MCS_LOBE_NODE) {
    mcs_lobe_query q = B;
    q.rpm_min = S0;
    q.rpm_max = S0 + MCS_LOBE_NODE;
    q.modal = (uint32_t)qs.size();
    qs.push_back(q);
    centre.push_back(S0 + MCS_LOBE_NODE / 2);
    begin.push_back((int)samples.size());
    for (double S = S0; S < std::min(hi, S0 + MCS_LOBE_NODE); S += MCS_LOBE_STEP)
      samples.push_back(S);
    count.push_back((int)samples.size() - begin.back());
  }
  *n_out = samples.size();
  if (!rpm_out) return MCS_OK;
  if (!alim_out) return fail(MCS_ERR_ARG, "alim is NULL");
  if (cap < samples.size())
    return fail(MCS_ERR_ARG, "the curve has %zu points, cap is %zu", samples.size(), cap);
  std::vector<mcs_modal> modals(qs.size());
  int rc = mcs_modes_at(sp, frfs, n_frfs, centre.data(), centre.size(), modals.data());
  if (rc) return rc;
  if (samples.empty()) return MCS_OK;
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  DevBuf dm, dq, dr, dout, db, dc;
  auto release = [&]() {
    dm.release(); dq.release(); dr.release(); dout.release(); db.release(); dc.release();
  };
  if ((rc = dm.ensure(sizeof(mcs_modal) * modals.size())) ||
      (rc = dq.ensure(sizeof(mcs_lobe_query) * qs.size())) ||
      (rc = dr.ensure(sizeof(double) * samples.size())) ||
      (rc = dout.ensure(sizeof(double) * samples.size())) ||
      (rc = db.ensure(sizeof(int) * qs.size())) || (rc = dc.ensure(sizeof(int) * qs.size()))) {
    release();
    return rc;
  }
  cudaStream_t st = c->stream;
  cudaError_t e = cudaMemcpyAsync(dm.p, modals.data(), sizeof(mcs_modal) * modals.size(),
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dq.p, qs.data(), sizeof(mcs_lobe_query) * qs.size(),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dr.p, samples.data(), sizeof(double) * samples.size(),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(db.p, begin.data(), sizeof(int) * qs.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dc.p, count.data(), sizeof(int) * qs.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = (cudaError_t)launch_lobes(st, static_cast<const mcs_modal*>(dm.p),
                                  static_cast<const mcs_lobe_query*>(dq.p), (int)qs.size(),
                                  static_cast<const double*>(dr.p), (int)samples.size(),
                                  static_cast<double*>(dout.p), static_cast<const int*>(db.p),
                                  static_cast<const int*>(dc.p));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(alim_out, dout.p, sizeof(double) * samples.size(),
                        cudaMemcpyDeviceToHost, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  release();
  if (e != cudaSuccess) return fail(MCS_ERR_CUDA, "composite lobes failed: %s", cudaGetErrorString(e));
  if (e2 != cudaSuccess) return fail(MCS_ERR_CUDA, "composite lobes failed: %s", cudaGetErrorString(e2));
  for (size_t i = 0; i < samples.size(); i++) {
    rpm_out[i] = samples[i];
    if (alim_out[i] == INFINITY) alim_out[i] = 1e3;  // sim.js:282
  }
  return MCS_OK;
}

int mcs_curve_alim(const double* cr, const double* ca, size_t n_curve, const double* rpm,
                   size_t n, double* out) {
  if ((n_curve && (!cr || !ca)) || (n && (!rpm || !out)))
    return fail(MCS_ERR_ARG, "NULL curve, speeds or output");
  bool ascending = true;
  for (size_t i = 1; i < n_curve; i++) ascending = ascending && cr[i] >= cr[i - 1];
  auto seg = [&](size_t i, double v, double& best) {  // segment [i-1, i] if it covers v
    if (v >= cr[i - 1] && v <= cr[i]) {
      const double span = cr[i] - cr[i - 1];
      const double t = (v - cr[i - 1]) / (span != 0 ? span : 1);
      best = std::min(best, ca[i - 1] + (ca[i] - ca[i - 1]) * t);
    }
  };
  for (size_t r = 0; r < n; r++) {
    const double v = rpm[r];
    double best = INFINITY;
    if (ascending) {  // the covering segments follow the first speed >= v
      const size_t first = (size_t)(std::lower_bound(cr, cr + n_curve, v) - cr);
      for (size_t i = std::max<size_t>(first, 1); i < n_curve && cr[i - 1] <= v; i++)
        seg(i, v, best);
    } else {
      for (size_t i = 1; i < n_curve; i++) seg(i, v, best);
    }
    out[r] = best;
  }
  return MCS_OK;
}

int mcs_measure_peaks(mcs_ctx* c, mcs_peaks* out) {
  if (!c || !out) return fail(MCS_ERR_ARG, "NULL ctx or output");
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  DevBuf scratch;
  int rc = scratch.ensure(16 << 10);
  if (rc) return rc;
  rc = measure_peaks(c->stream, c->sms, scratch.p, &out->fp32_tflops, &out->fp64_tflops,
                     &out->smem_tbps);
  cudaStreamSynchronize(c->stream);
  scratch.release();
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free solve
// mcs_solve without device allocations: the per-point parameters, the work order, the
// queue counter and the device copy of the results sit in this file-scope array, which
// every device that loads the library keeps until exit.  Host code must not use the
// array's name as an address: its device address is looked up once per device with
// cudaGetSymbolAddress and passed to the kernels.
namespace {

constexpr size_t kNaMax = MCS_NOALLOC_MAX_POINTS;
constexpr size_t kNaAlign = 256;
constexpr size_t na_up(size_t b) { return (b + kNaAlign - 1) & ~(kNaAlign - 1); }
constexpr size_t kNaQueueOff = 0;
constexpr size_t kNaOrderOff = kNaAlign;
constexpr size_t kNaParamsOff = kNaOrderOff + na_up(sizeof(int32_t) * kNaMax);
constexpr size_t kNaResultsOff = kNaParamsOff + na_up(sizeof(PointParams) * kNaMax);
constexpr size_t kNaBytes = kNaResultsOff + na_up(sizeof(mcs_result) * kNaMax);
constexpr int kNaMaxDevices = 64;
constexpr int kNaChunk = 32;  // points prepared per host-to-device copy (on the stack)

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

std::mutex g_na_setup_mu;
unsigned char* g_na_ptr[kNaMaxDevices] = {};
std::mutex g_na_dev_mu[kNaMaxDevices];

// Device address of the scratch array on the current device (looked up on first use).
int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kNaMaxDevices)
    return fail(MCS_ERR_UNSUPPORTED, "device %d: the allocation-free path serves devices "
                "0..%d", device, kNaMaxDevices - 1);
  std::lock_guard<std::mutex> lk(g_na_setup_mu);
  if (!g_na_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(MCS_ERR_CUDA, "cudaGetSymbolAddress of the scratch area failed: %s",
                  cudaGetErrorString(e));
    g_na_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_na_ptr[device];
  return MCS_OK;
}

}  // namespace

extern "C" int mcs_solve_noalloc(mcs_ctx* c, const mcs_setup* setups, size_t n_setups,
                                 const mcs_modal* modals, size_t n_modals,
                                 const mcs_point* points, size_t n_points, const mcs_opts* o,
                                 mcs_result* out) {
  if (!c) return fail(MCS_ERR_ARG, "ctx is NULL");
  if (n_points && !out) return fail(MCS_ERR_ARG, "out is NULL");
  if (n_points > kNaMax)
    return fail(MCS_ERR_ARG, "%zu points exceed the %zu the preallocated scratch area holds "
                "(MCS_NOALLOC_MAX_POINTS); split the batch or use mcs_solve",
                n_points, kNaMax);
  std::lock_guard<std::mutex> lk(c->mu);
  MCS_CUDA(cudaSetDevice(c->device));
  int rc = check_inputs(setups, n_setups, modals, n_modals, points, n_points, o);
  if (rc) return rc;
  if (n_points == 0) return MCS_OK;
  unsigned char* base = nullptr;
  if ((rc = noalloc_scratch(c->device, &base))) return rc;
  std::lock_guard<std::mutex> dev_lk(g_na_dev_mu[c->device]);
  cudaStream_t st = c->stream;
  auto* d_queue = reinterpret_cast<unsigned int*>(base + kNaQueueOff);
  auto* d_order = reinterpret_cast<int32_t*>(base + kNaOrderOff);
  auto* d_params = reinterpret_cast<PointParams*>(base + kNaParamsOff);
  auto* d_results = reinterpret_cast<mcs_result*>(base + kNaResultsOff);

  // Everything that touches the scratch area; whatever it returns, the stream is drained
  // below before the device lock is released, so that no copy or kernel of this call is
  // still using the area when the next call starts, on this context or another.
  auto body = [&]() -> int {
    // prepare on the host in stack-sized chunks and copy each into the scratch area
    PointParams chunk[kNaChunk];
    double cost[kNaMax];
    int32_t order[kNaMax];
    int smem = 0, slots = 1, modes = 1, nl = 0, gr = 0;
    for (size_t i0 = 0; i0 < n_points; i0 += kNaChunk) {
      const size_t m = std::min<size_t>(kNaChunk, n_points - i0);
      for (size_t j = 0; j < m; j++) {
        const size_t i = i0 + j;
        Prepared pr;
        const int prc = prepare_point(setups[points[i].setup], modals[points[i].modal],
                                      points[i].S, *o, o->a_max, pr);
        if (prc) return fail(prc, "point %zu: %s", i, g_last_error.c_str());
        chunk[j] = pr.pp;
        cost[i] = pr.cost;
        smem = std::max(smem, pr.pp.smem_bytes);
        slots = std::max(slots, slots_for(pr.pp.nz_max));
        modes = std::max(modes, pr.modes);
        nl = std::max(nl, pr.nl);
        gr = std::max(gr, pr.pp.groups > 1 ? 1 : 0);
      }
      MCS_CUDA(cudaMemcpyAsync(d_params + i0, chunk, sizeof(PointParams) * m,
                               cudaMemcpyHostToDevice, st));
      MCS_CUDA(cudaStreamSynchronize(st));  // the chunk buffer is reused
    }
    // largest first, for the persistent warps' load balance
    for (size_t i = 0; i < n_points; i++) order[i] = (int32_t)i;
    std::sort(order, order + n_points, [&](int32_t a, int32_t b) { return cost[a] > cost[b]; });
    MCS_CUDA(cudaMemcpyAsync(d_order, order, sizeof(int32_t) * n_points,
                             cudaMemcpyHostToDevice, st));
    // the queue counter must start at zero; the area keeps the previous call's contents
    MCS_CUDA(cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st));
    const KernelShape shape{slots, modes, o->precision == MCS_FP64 ? 1 : 0, nl, gr};
    smem = (smem + 15) & ~15;
    int bps = 0;
    const int orc = occupancy_solve(shape, smem, &bps);
    if (orc != 0)
      return fail(MCS_ERR_CUDA, "occupancy query failed: %s",
                  cudaGetErrorString((cudaError_t)orc));
    if (bps < 1) return fail(MCS_ERR_UNSUPPORTED, "a %d-byte warp does not fit on an SM", smem);
    const int grid = (int)std::min<long long>((long long)n_points, (long long)bps * c->sms);
    const int lrc = launch_solve(shape, grid, smem, st, d_params, d_order, (int)n_points,
                                 dev_opts(o), d_results, d_queue, nullptr, nullptr);
    if (lrc != 0)
      return fail(MCS_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString((cudaError_t)lrc));
    MCS_CUDA(cudaMemcpyAsync(out, d_results, sizeof(mcs_result) * n_points,
                             cudaMemcpyDeviceToHost, st));
    return MCS_OK;
  };
  rc = body();
  const cudaError_t e = cudaStreamSynchronize(st);
  if (!rc && e != cudaSuccess)
    rc = fail(MCS_ERR_CUDA, "allocation-free solve failed: %s", cudaGetErrorString(e));
  return rc;
}
