/*
 * Drives the mcs.node glue (machinig-sim_b200/node/mcs_napi.c) through the fake Node-API
 * runtime with the reference's argument objects, printing one JSON line per case:
 *   {"case": name, "threw": code, "message": text}   or   {"case": name, ...values}
 * Usage: driver <modal k [N/mm]> <modal fn [Hz]>
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "fake_napi.h"

napi_value napi_register_module_v1(napi_env env, napi_value exports);

static napi_value exports_;

static napi_value tool(double N, double R, double runout) {
  napi_value t = fk_obj();
  fk_set(t, "N", fk_num(N));
  if (R > 0) fk_set(t, "R", fk_num(R));
  else fk_set(t, "D", fk_num(10));
  fk_set(t, "helixDeg", fk_num(30));
  fk_set(t, "type", fk_str("flat"));
  fk_set(t, "fluteLen", fk_num(25));
  if (runout > 0) fk_set(t, "runout", fk_num(runout));
  return t;
}

static napi_value s50c(void) {
  napi_value m = fk_obj();
  fk_set(m, "Ktc", fk_num(2100));
  fk_set(m, "Krc", fk_num(850));
  fk_set(m, "Kte", fk_num(35));
  fk_set(m, "Kre", fk_num(45));
  fk_set(m, "mc", fk_num(0.14));
  fk_set(m, "Ci", fk_num(1.5e5));
  return m;
}

static napi_value modal(double k, double fn) {
  napi_value m = fk_obj();
  fk_set(m, "k", fk_num(k));
  fk_set(m, "fn", fk_num(fn));
  fk_set(m, "zeta", fk_num(0.04));
  return m;
}

static napi_value arc(void) {
  napi_value a = fk_arr();
  fk_push(a, fk_num(M_PI / 2));
  fk_push(a, fk_num(M_PI));
  return a;
}

static napi_value opts(double revs, double iters, const char* precision) {
  napi_value o = fk_obj();
  if (revs > 0) fk_set(o, "revs", fk_num(revs));
  if (iters > 0) fk_set(o, "iters", fk_num(iters));
  if (precision) fk_set(o, "precision", fk_str(precision));
  return o;
}

/* prints the thrown error, if any; returns 1 when the call threw */
static int threw(const char* name) {
  if (!g_env.exception) return 0;
  napi_value c = fk_get(g_env.exception, "code"), m = fk_get(g_env.exception, "message");
  printf("{\"case\": \"%s\", \"threw\": \"%s\", \"message\": \"%s\"}\n", name,
         c ? c->s : "", m ? m->s : "");
  return 1;
}

static void print_promise(const char* name, napi_value p) {
  napi_value v = fk_get(p, "value");
  if (p->b == 2) {
    napi_value c = fk_get(v, "code"), m = fk_get(v, "message");
    printf("{\"case\": \"%s\", \"rejected\": \"%s\", \"message\": \"%s\"}\n", name,
           c ? c->s : "", m ? m->s : "");
    return;
  }
  printf("{\"case\": \"%s\", \"state\": %d, \"S\": [", name, p->b);
  for (int i = 0; v && i < v->len; i++)
    printf("%s%.17g", i ? ", " : "", fk_get(v->elems[i], "S")->num);
  printf("], \"alim\": [");
  for (int i = 0; v && i < v->len; i++)
    printf("%s%.17g", i ? ", " : "", fk_get(v->elems[i], "alim")->num);
  printf("], \"open\": [");
  for (int i = 0; v && i < v->len; i++)
    printf("%s%d", i ? ", " : "", fk_get(v->elems[i], "open")->b);
  printf("]}\n");
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const double k = atof(argv[1]), fn = atof(argv[2]);
  exports_ = fk_obj();
  napi_register_module_v1(&g_env, exports_);

  /* argument errors are thrown before any device work */
  {
    napi_value a[3] = {tool(3, 5, 0), modal(k, fn), s50c()};
    fk_call(exports_, "chatterAt", 3, a);
    threw("missing_args");
  }
  {
    napi_value a[7] = {tool(0, 5, 0), modal(k, fn), s50c(), fk_num(8000), arc(), fk_num(0.05),
                       opts(30, 6, NULL)};
    fk_call(exports_, "timeDomainLimit", 7, a);
    threw("bad_tool");
  }
  {
    napi_value m = fk_obj(), xs = fk_arr();
    for (int i = 0; i < 5; i++) fk_push(xs, modal(k, fn));
    fk_set(m, "modesX", xs);
    napi_value a[7] = {tool(3, 5, 0), m, s50c(), fk_num(8000), arc(), fk_num(0.05),
                       opts(30, 6, NULL)};
    fk_call(exports_, "timeDomainLimit", 7, a);
    threw("bad_modal");
  }
  /* computations (on a machine without a device these throw MCS_ERR_CUDA) */
  {
    napi_value a[7] = {tool(3, 5, 0), modal(k, fn), s50c(), fk_num(8000), arc(), fk_num(0.05),
                       opts(0, 0, "fp64")};
    napi_value r = fk_call(exports_, "timeDomainLimit", 7, a);
    if (!threw("tdl_defaults_fp64")) {
      napi_value b = fk_get(r, "bracket");
      printf("{\"case\": \"tdl_defaults_fp64\", \"alim\": %.17g, \"lo\": %.17g, \"hi\": %.17g}\n",
             fk_get(r, "alim")->num, b->elems[0]->num, b->elems[1]->num);
    }
  }
  {
    napi_value a[7] = {tool(3, 0, 5), modal(k, fn), s50c(), fk_num(8000), arc(), fk_num(0.05),
                       opts(30, 6, NULL)};
    napi_value r = fk_call(exports_, "timeDomainLimit", 7, a);
    if (!threw("tdl_D_runout"))
      printf("{\"case\": \"tdl_D_runout\", \"alim\": %.17g, \"open\": %d}\n",
             fk_get(r, "alim")->num, isinf(fk_get(r, "bracket")->elems[1]->num) ? 1 : 0);
  }
  {
    napi_value o = opts(30, 6, NULL);
    fk_set(o, "aMax", fk_num(0.3));
    napi_value a[7] = {tool(3, 5, 0), modal(k, fn), s50c(), fk_num(8000), arc(), fk_num(0.05), o};
    napi_value r = fk_call(exports_, "timeDomainLimit", 7, a);
    if (!threw("tdl_open"))
      printf("{\"case\": \"tdl_open\", \"alim\": %.17g, \"hi_inf\": %d}\n",
             fk_get(r, "alim")->num, isinf(fk_get(r, "bracket")->elems[1]->num) ? 1 : 0);
  }
  for (int i = 0; i < 2; i++) {
    const double ap = i ? 3.0 : 0.3;
    napi_value a[8] = {tool(3, 5, 0), modal(k, fn), s50c(), fk_num(8000), arc(), fk_num(0.05),
                       fk_num(ap), opts(60, 0, NULL)};
    napi_value r = fk_call(exports_, "chatterAt", 8, a);
    if (!threw(i ? "chatter_deep" : "chatter_shallow"))
      printf("{\"case\": \"%s\", \"chatter\": %d}\n", i ? "chatter_deep" : "chatter_shallow",
             r->b);
  }
  {
    napi_value pts = fk_arr();
    const double speeds[3] = {6000, 9000, 13000};
    for (int i = 0; i < 3; i++) {
      napi_value p = fk_obj();
      fk_set(p, "S", fk_num(speeds[i]));
      fk_set(p, "modal", modal(k, fn));
      fk_push(pts, p);
    }
    napi_value a[6] = {tool(3, 5, 0), s50c(), arc(), fk_num(0.05), pts, opts(30, 6, NULL)};
    napi_value p = fk_call(exports_, "timeDomainLimits", 6, a);
    if (!threw("sweep")) print_promise("sweep", p);
  }
  {
    napi_value prm = modal(k, fn), rpms = fk_arr();
    fk_set(prm, "N", fk_num(3));
    fk_set(prm, "Ktc", fk_num(2100));
    fk_set(prm, "Krc", fk_num(850));
    fk_set(prm, "phiSt", fk_num(M_PI / 2));
    fk_set(prm, "phiEx", fk_num(M_PI));
    fk_set(prm, "lobes", fk_num(30));
    fk_set(prm, "rpmMin", fk_num(2000));
    fk_set(prm, "rpmMax", fk_num(40000));
    fk_push(rpms, fk_num(2500));
    fk_push(rpms, fk_num(8000));
    napi_value a[2] = {prm, rpms};
    napi_value r = fk_call(exports_, "lobeLimit", 2, a);
    if (!threw("lobes")) {
      const double* d = (const double*)r->data;
      printf("{\"case\": \"lobes\", \"alim\": [%.17g, %.17g]}\n", d[0], d[1]);
    }
  }
  return 0;
}
