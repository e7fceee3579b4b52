/*
 * Node-API addon over libmcs.so: the reference's stability functions for JavaScript hosts
 * (Node, Electron), same names, arguments and return shapes as src/stabtd.js and
 * src/sld.js.  Argument objects are the reference's:
 *
 *   tool  {N, R | D, helixDeg, type, fluteLen, runout [um], runoutPhase}
 *   modal {k, fn, zeta, modesX?, modesY?}       mat {Ktc, Krc, Kte, Kre, mc, Ci}
 *   opts  {aMin, aMax, iters, revs, nonlinear} + honorRunout, stepsPerTooth, slices,
 *         chatterIdx, precision ('fp32' | 'fp64')
 *
 * Exports
 *   chatterAt(tool, modal, mat, S, arc, fz, ap, opts?)       -> boolean    (stabtd.js:14)
 *   chatterIndex(tool, modal, mat, S, arc, fz, ap, opts?)    -> {index, amp, once}
 *   timeDomainLimit(tool, modal, mat, S, arc, fz, opts?)     -> {alim, bracket} (stabtd.js:24)
 *   timeDomainLimits(tool, mat, arc, fz, points, opts?)      -> Promise<[{S, alim, open}]>
 *       the Worker's sweep (stabworker.js:8-13) as one asynchronous GPU job
 *   cancelSweeps()                                           -> number of jobs cancelled
 *   lobeLimit(params, rpms)                                  -> Float64Array (sld.js:23,64)
 *
 * A failing call throws an Error whose code is the mcs_status name and whose message is
 * mcs_last_error(); a cancelled sweep rejects with code MCS_ERR_CANCELLED.
 */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/mcs.h"
#include "napi_min.h"

#define MAX_ARGS 8
#define MAX_JOBS 64

static mcs_ctx* g_ctx = NULL;
static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
static mcs_job* g_jobs[MAX_JOBS];

static const char* status_name(int st) {
  switch (st) {
    case MCS_OK: return "MCS_OK";
    case MCS_ERR_ARG: return "MCS_ERR_ARG";
    case MCS_ERR_CUDA: return "MCS_ERR_CUDA";
    case MCS_ERR_TIMEOUT: return "MCS_ERR_TIMEOUT";
    case MCS_ERR_DIVERGED: return "MCS_ERR_DIVERGED";
    case MCS_ERR_CANCELLED: return "MCS_ERR_CANCELLED";
    case MCS_ERR_NOMEM: return "MCS_ERR_NOMEM";
    case MCS_ERR_UNSUPPORTED: return "MCS_ERR_UNSUPPORTED";
    default: return "MCS_ERR_STATE";
  }
}

static napi_value throw_status(napi_env env, int st) {
  napi_throw_error(env, status_name(st), mcs_last_error());
  return NULL;
}

static napi_value throw_arg(napi_env env, const char* msg) {
  napi_throw_error(env, "MCS_ERR_ARG", msg);
  return NULL;
}

/* The process-wide context, on the device named by MCS_DEVICE (default 0). */
static int context(mcs_ctx** out) {
  int st = MCS_OK;
  pthread_mutex_lock(&g_mu);
  if (!g_ctx) {
    const char* d = getenv("MCS_DEVICE");
    st = mcs_create(&g_ctx, d ? atoi(d) : 0);
  }
  *out = g_ctx;
  pthread_mutex_unlock(&g_mu);
  return st;
}

/* ---- reading the reference's argument objects ---- */

static int has(napi_env env, napi_value obj, const char* name) {
  bool b = false;
  napi_valuetype t;
  if (!obj || napi_typeof(env, obj, &t) != napi_ok || t != napi_object) return 0;
  if (napi_has_named_property(env, obj, name, &b) != napi_ok || !b) return 0;
  napi_value v;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return 0;
  return napi_typeof(env, v, &t) == napi_ok && t != napi_undefined && t != napi_null;
}

/* number property; def when absent; -1 when present but not a number */
static int num(napi_env env, napi_value obj, const char* name, double def, double* out) {
  if (!has(env, obj, name)) {
    *out = def;
    return 0;
  }
  napi_value v;
  napi_get_named_property(env, obj, name, &v);
  return napi_get_value_double(env, v, out) == napi_ok ? 0 : -1;
}

static int boolean(napi_env env, napi_value obj, const char* name, int def, int* out) {
  if (!has(env, obj, name)) {
    *out = def;
    return 0;
  }
  napi_value v;
  bool b;
  napi_get_named_property(env, obj, name, &v);
  if (napi_get_value_bool(env, v, &b) != napi_ok) {
    double d; /* accept 0/1 as the JS truthiness of numbers */
    if (napi_get_value_double(env, v, &d) != napi_ok) return -1;
    b = d != 0;
  }
  *out = b ? 1 : 0;
  return 0;
}

static int str(napi_env env, napi_value obj, const char* name, char* buf, size_t n) {
  buf[0] = 0;
  if (!has(env, obj, name)) return 0;
  napi_value v;
  size_t len;
  napi_get_named_property(env, obj, name, &v);
  return napi_get_value_string_utf8(env, v, buf, n, &len) == napi_ok ? 0 : -1;
}

static int parse_tool(napi_env env, napi_value v, mcs_tool* t) {
  double N, R, D, helix, flute, runout, phase;
  char type[16];
  memset(t, 0, sizeof(*t));
  if (num(env, v, "N", NAN, &N) || num(env, v, "D", NAN, &D) || num(env, v, "R", D / 2, &R) ||
      num(env, v, "helixDeg", 30, &helix) || num(env, v, "fluteLen", 25, &flute) ||
      num(env, v, "runout", 0, &runout) || num(env, v, "runoutPhase", 0, &phase) ||
      str(env, v, "type", type, sizeof(type)))
    return -1;
  if (!(N >= 1 && N == floor(N)) || !(R > 0)) return -1;
  t->N = (int32_t)N;
  t->type = strcmp(type, "ball") == 0 ? MCS_TOOL_BALL : MCS_TOOL_FLAT;
  t->R = R;
  t->helix_deg = helix;
  t->flute_len = flute;
  t->runout = runout / 1000.0; /* um -> mm, the engine's unit (cutting.js:43) */
  t->runout_phase = phase;
  return 0;
}

static int parse_modes(napi_env env, napi_value obj, const char* name, mcs_mode* out, int* n) {
  *n = 0;
  if (!has(env, obj, name)) return 0;
  napi_value arr;
  bool isarr = false;
  uint32_t len = 0;
  napi_get_named_property(env, obj, name, &arr);
  if (napi_is_array(env, arr, &isarr) != napi_ok || !isarr) return -1;
  napi_get_array_length(env, arr, &len);
  if (len > MCS_MAX_MODES) return -1;
  for (uint32_t i = 0; i < len; i++) {
    napi_value m;
    napi_get_element(env, arr, i, &m);
    if (num(env, m, "k", NAN, &out[i].k) || num(env, m, "fn", NAN, &out[i].fn) ||
        num(env, m, "zeta", NAN, &out[i].zeta))
      return -1;
  }
  *n = (int)len;
  return 0;
}

/* modeSet (frf.js:6-11): x = modesX or the single mode, y = modesY or x */
static int parse_modal(napi_env env, napi_value v, mcs_modal* m) {
  memset(m, 0, sizeof(*m));
  int nx, ny;
  if (parse_modes(env, v, "modesX", m->x, &nx) || parse_modes(env, v, "modesY", m->y, &ny))
    return -1;
  if (nx == 0) {
    if (num(env, v, "k", NAN, &m->x[0].k) || num(env, v, "fn", NAN, &m->x[0].fn) ||
        num(env, v, "zeta", NAN, &m->x[0].zeta))
      return -1;
    nx = 1;
  }
  m->nx = nx;
  m->ny = ny;
  return 0;
}

static int parse_mat(napi_env env, napi_value v, mcs_material* m) {
  return num(env, v, "Ktc", NAN, &m->Ktc) || num(env, v, "Krc", NAN, &m->Krc) ||
                 num(env, v, "Kte", 0, &m->Kte) || num(env, v, "Kre", 0, &m->Kre) ||
                 num(env, v, "mc", 0, &m->mc) || num(env, v, "Ci", 0, &m->Ci)
             ? -1
             : 0;
}

static int parse_opts(napi_env env, napi_value v, mcs_opts* o) {
  double iters, revs, spt, slices;
  char prec[8];
  mcs_default_opts(o);
  if (num(env, v, "aMin", o->a_min, &o->a_min) || num(env, v, "aMax", o->a_max, &o->a_max) ||
      num(env, v, "iters", o->iters, &iters) || num(env, v, "revs", o->revs, &revs) ||
      boolean(env, v, "nonlinear", 1, &o->nonlinear) ||
      boolean(env, v, "honorRunout", 0, &o->honor_runout) ||
      num(env, v, "stepsPerTooth", 0, &spt) || num(env, v, "slices", 0, &slices) ||
      num(env, v, "chatterIdx", o->chatter_idx, &o->chatter_idx) ||
      str(env, v, "precision", prec, sizeof(prec)))
    return -1;
  o->iters = (int32_t)iters;
  o->revs = (int32_t)revs;
  o->steps_per_tooth = (int32_t)spt;
  o->slices = (int32_t)slices;
  /* no precision given: the library's default (FP64, the reference's arithmetic) */
  if (strcmp(prec, "fp32") == 0)
    o->precision = MCS_FP32;
  else if (strcmp(prec, "fp64") == 0)
    o->precision = MCS_FP64;
  else if (prec[0] != 0)
    return -1;
  return 0;
}

static int arc_of(napi_env env, napi_value v, double* st, double* ex) {
  bool isarr = false;
  uint32_t len = 0;
  napi_value a, b;
  if (napi_is_array(env, v, &isarr) != napi_ok || !isarr) return -1;
  napi_get_array_length(env, v, &len);
  if (len < 2) return -1;
  napi_get_element(env, v, 0, &a);
  napi_get_element(env, v, 1, &b);
  return napi_get_value_double(env, a, st) == napi_ok &&
                 napi_get_value_double(env, b, ex) == napi_ok
             ? 0
             : -1;
}

static napi_value number(napi_env env, double d) {
  napi_value v;
  napi_create_double(env, d, &v);
  return v;
}

/* one setup + one modal + one point from the positional arguments (tool, modal, mat, S,
 * arc, fz) */
static int one_point(napi_env env, napi_value* argv, mcs_setup* s, mcs_modal* m, mcs_point* p) {
  double S;
  memset(s, 0, sizeof(*s));
  if (parse_tool(env, argv[0], &s->tool) || parse_modal(env, argv[1], m) ||
      parse_mat(env, argv[2], &s->mat) || napi_get_value_double(env, argv[3], &S) != napi_ok ||
      arc_of(env, argv[4], &s->arc_st, &s->arc_ex) ||
      napi_get_value_double(env, argv[5], &s->fz) != napi_ok)
    return -1;
  p->setup = 0;
  p->modal = 0;
  p->S = S;
  return 0;
}

static napi_value trial(napi_env env, napi_callback_info info, int want_index) {
  size_t argc = MAX_ARGS;
  napi_value argv[MAX_ARGS];
  napi_get_cb_info(env, info, &argc, argv, NULL, NULL);
  if (argc < 7) return throw_arg(env, "chatterAt(tool, modal, mat, S, arc, fz, ap, opts?)");
  mcs_setup s;
  mcs_modal m;
  mcs_point p;
  mcs_opts o;
  mcs_trial t = {0, 0, 0.0};
  if (one_point(env, argv, &s, &m, &p) ||
      napi_get_value_double(env, argv[6], &t.ap) != napi_ok ||
      parse_opts(env, argc > 7 ? argv[7] : NULL, &o))
    return throw_arg(env, "invalid argument object");
  mcs_ctx* ctx;
  int st = context(&ctx);
  if (st) return throw_status(env, st);
  mcs_trial_result r;
  st = mcs_chatter_at(ctx, &s, 1, &m, 1, &p, 1, &t, 1, &o, &r);
  if (st) return throw_status(env, st);
  if (!want_index) {
    napi_value b;
    napi_get_boolean(env, r.chatter != 0, &b);
    return b;
  }
  napi_value obj;
  napi_create_object(env, &obj);
  napi_set_named_property(env, obj, "index", number(env, r.index));
  napi_set_named_property(env, obj, "amp", number(env, r.amp));
  napi_set_named_property(env, obj, "once", number(env, r.once));
  return obj;
}

static napi_value js_chatter_at(napi_env env, napi_callback_info info) {
  return trial(env, info, 0);
}
static napi_value js_chatter_index(napi_env env, napi_callback_info info) {
  return trial(env, info, 1);
}

static napi_value js_time_domain_limit(napi_env env, napi_callback_info info) {
  size_t argc = MAX_ARGS;
  napi_value argv[MAX_ARGS];
  napi_get_cb_info(env, info, &argc, argv, NULL, NULL);
  if (argc < 6) return throw_arg(env, "timeDomainLimit(tool, modal, mat, S, arc, fz, opts?)");
  mcs_setup s;
  mcs_modal m;
  mcs_point p;
  mcs_opts o;
  if (one_point(env, argv, &s, &m, &p) || parse_opts(env, argc > 6 ? argv[6] : NULL, &o))
    return throw_arg(env, "invalid argument object");
  mcs_ctx* ctx;
  int st = context(&ctx);
  if (st) return throw_status(env, st);
  mcs_result r;
  st = mcs_solve(ctx, &s, 1, &m, 1, &p, 1, &o, &r);
  if (st) return throw_status(env, st);
  if (r.status != MCS_OK && r.status != MCS_ERR_DIVERGED) return throw_status(env, r.status);
  napi_value obj, bracket;
  napi_create_object(env, &obj);
  napi_create_array_with_length(env, 2, &bracket);
  napi_set_element(env, bracket, 0, number(env, r.lo));
  napi_set_element(env, bracket, 1, number(env, r.open ? INFINITY : r.hi));
  napi_set_named_property(env, obj, "alim", number(env, r.alim));
  napi_set_named_property(env, obj, "bracket", bracket);
  return obj;
}

/* ---- the asynchronous sweep ---- */
typedef struct {
  napi_async_work work;
  napi_deferred deferred;
  mcs_setup setup;
  mcs_modal* modals;
  mcs_point* points;
  mcs_result* out;
  size_t n;
  mcs_opts opts;
  mcs_job* job;
  int status;
  char error[256];
} sweep_t;

static void sweep_register(mcs_job* j, int add) {
  pthread_mutex_lock(&g_mu);
  for (int i = 0; i < MAX_JOBS; i++) {
    if (add && !g_jobs[i]) {
      g_jobs[i] = j;
      break;
    }
    if (!add && g_jobs[i] == j) {
      g_jobs[i] = NULL;
      break;
    }
  }
  pthread_mutex_unlock(&g_mu);
}

static void sweep_execute(napi_env env, void* data) {
  (void)env;
  sweep_t* w = (sweep_t*)data;
  mcs_ctx* ctx;
  w->status = context(&ctx);
  if (w->status == MCS_OK)
    w->status = mcs_solve_async(ctx, &w->setup, 1, w->modals, w->n, w->points, w->n, &w->opts,
                                w->out, &w->job);
  if (w->status == MCS_OK) {
    sweep_register(w->job, 1);
    w->status = mcs_job_wait(w->job);
    sweep_register(w->job, 0);
  }
  if (w->status) snprintf(w->error, sizeof(w->error), "%s", mcs_last_error());
}

static void sweep_complete(napi_env env, napi_status status, void* data) {
  sweep_t* w = (sweep_t*)data;
  if (status != napi_ok && w->status == MCS_OK) w->status = MCS_ERR_STATE;
  if (w->status) {
    napi_value code, msg, err;
    napi_create_string_utf8(env, status_name(w->status), (size_t)-1, &code);
    napi_create_string_utf8(env, w->error, (size_t)-1, &msg);
    napi_create_error(env, code, msg, &err);
    napi_set_named_property(env, err, "code", code);
    napi_reject_deferred(env, w->deferred, err);
  } else {
    napi_value arr;
    napi_create_array_with_length(env, w->n, &arr);
    for (size_t i = 0; i < w->n; i++) {
      napi_value o, open;
      napi_create_object(env, &o);
      napi_get_boolean(env, w->out[i].open != 0, &open);
      napi_set_named_property(env, o, "S", number(env, w->points[i].S));
      napi_set_named_property(env, o, "alim", number(env, w->out[i].alim));
      napi_set_named_property(env, o, "open", open);
      napi_set_element(env, arr, (uint32_t)i, o);
    }
    napi_resolve_deferred(env, w->deferred, arr);
  }
  if (w->job) mcs_job_free(w->job);
  napi_delete_async_work(env, w->work);
  free(w->modals);
  free(w->points);
  free(w->out);
  free(w);
}

static napi_value js_time_domain_limits(napi_env env, napi_callback_info info) {
  size_t argc = MAX_ARGS;
  napi_value argv[MAX_ARGS];
  napi_get_cb_info(env, info, &argc, argv, NULL, NULL);
  if (argc < 5) return throw_arg(env, "timeDomainLimits(tool, mat, arc, fz, points, opts?)");
  bool isarr = false;
  uint32_t n = 0;
  if (napi_is_array(env, argv[4], &isarr) != napi_ok || !isarr)
    return throw_arg(env, "points must be an array of {S, modal}");
  napi_get_array_length(env, argv[4], &n);
  sweep_t* w = (sweep_t*)calloc(1, sizeof(sweep_t));
  if (!w) return throw_status(env, MCS_ERR_NOMEM);
  w->n = n;
  w->modals = (mcs_modal*)calloc(n ? n : 1, sizeof(mcs_modal));
  w->points = (mcs_point*)calloc(n ? n : 1, sizeof(mcs_point));
  w->out = (mcs_result*)calloc(n ? n : 1, sizeof(mcs_result));
  int bad = !w->modals || !w->points || !w->out;
  bad = bad || parse_tool(env, argv[0], &w->setup.tool) || parse_mat(env, argv[1], &w->setup.mat) ||
        arc_of(env, argv[2], &w->setup.arc_st, &w->setup.arc_ex) ||
        napi_get_value_double(env, argv[3], &w->setup.fz) != napi_ok ||
        parse_opts(env, argc > 5 ? argv[5] : NULL, &w->opts);
  for (uint32_t i = 0; !bad && i < n; i++) {
    napi_value p, mv;
    napi_get_element(env, argv[4], i, &p);
    bad = num(env, p, "S", NAN, &w->points[i].S) || !has(env, p, "modal");
    if (!bad) {
      napi_get_named_property(env, p, "modal", &mv);
      bad = parse_modal(env, mv, &w->modals[i]);
    }
    w->points[i].setup = 0;
    w->points[i].modal = i;
  }
  if (bad) {
    free(w->modals);
    free(w->points);
    free(w->out);
    free(w);
    return throw_arg(env, "invalid argument object");
  }
  napi_value promise, name;
  napi_create_promise(env, &w->deferred, &promise);
  napi_create_string_utf8(env, "mcs.timeDomainLimits", (size_t)-1, &name);
  napi_create_async_work(env, NULL, name, sweep_execute, sweep_complete, w, &w->work);
  napi_queue_async_work(env, w->work);
  return promise;
}

static napi_value js_cancel_sweeps(napi_env env, napi_callback_info info) {
  (void)info;
  int n = 0;
  pthread_mutex_lock(&g_mu);
  for (int i = 0; i < MAX_JOBS; i++)
    if (g_jobs[i] && mcs_job_cancel(g_jobs[i]) == MCS_OK) n++;
  pthread_mutex_unlock(&g_mu);
  return number(env, n);
}

static napi_value js_lobe_limit(napi_env env, napi_callback_info info) {
  size_t argc = MAX_ARGS;
  napi_value argv[MAX_ARGS];
  napi_get_cb_info(env, info, &argc, argv, NULL, NULL);
  if (argc < 2) return throw_arg(env, "lobeLimit(params, rpms)");
  mcs_modal m;
  mcs_lobe_query q;
  double N, lobes;
  memset(&q, 0, sizeof(q));
  if (parse_modal(env, argv[0], &m) || num(env, argv[0], "N", NAN, &N) ||
      num(env, argv[0], "lobes", 8, &lobes) || num(env, argv[0], "Ktc", NAN, &q.Ktc) ||
      num(env, argv[0], "Krc", NAN, &q.Krc) || num(env, argv[0], "phiSt", NAN, &q.phi_st) ||
      num(env, argv[0], "phiEx", NAN, &q.phi_ex) ||
      num(env, argv[0], "rpmMin", 1000, &q.rpm_min) ||
      num(env, argv[0], "rpmMax", 40000, &q.rpm_max))
    return throw_arg(env, "invalid lobe parameters");
  q.N = (int32_t)N;
  q.lobes = (int32_t)lobes;
  bool isarr = false;
  uint32_t n = 0;
  if (napi_is_array(env, argv[1], &isarr) != napi_ok || !isarr)
    return throw_arg(env, "rpms must be an array of numbers");
  napi_get_array_length(env, argv[1], &n);
  double* rpm = (double*)calloc(n ? n : 1, sizeof(double));
  if (!rpm) return throw_status(env, MCS_ERR_NOMEM);
  for (uint32_t i = 0; i < n; i++) {
    napi_value e;
    napi_get_element(env, argv[1], i, &e);
    if (napi_get_value_double(env, e, &rpm[i]) != napi_ok) {
      free(rpm);
      return throw_arg(env, "rpms must be numbers");
    }
  }
  napi_value ab, ta;
  void* data = NULL;
  napi_create_arraybuffer(env, (size_t)n * sizeof(double), &data, &ab);
  mcs_ctx* ctx;
  int st = context(&ctx);
  if (!st && n) st = mcs_lobes_alim(ctx, &m, 1, &q, 1, rpm, n, (double*)data);
  free(rpm);
  if (st) return throw_status(env, st);
  napi_create_typedarray(env, napi_float64_array, n, ab, 0, &ta);
  return ta;
}

napi_value napi_register_module_v1(napi_env env, napi_value exports) {
  const napi_property_descriptor props[] = {
      {"chatterAt", NULL, js_chatter_at, NULL, NULL, NULL, napi_enumerable, NULL},
      {"chatterIndex", NULL, js_chatter_index, NULL, NULL, NULL, napi_enumerable, NULL},
      {"timeDomainLimit", NULL, js_time_domain_limit, NULL, NULL, NULL, napi_enumerable, NULL},
      {"timeDomainLimits", NULL, js_time_domain_limits, NULL, NULL, NULL, napi_enumerable, NULL},
      {"cancelSweeps", NULL, js_cancel_sweeps, NULL, NULL, NULL, napi_enumerable, NULL},
      {"lobeLimit", NULL, js_lobe_limit, NULL, NULL, NULL, napi_enumerable, NULL},
  };
  napi_define_properties(env, exports, sizeof(props) / sizeof(props[0]), props);
  return exports;
}
