/*
 * A minimal stand-in for the Node-API runtime, for testing the mcs.node glue without a
 * JavaScript engine (none exists in this image).  It implements the functions the addon
 * declares in napi_min.h over a tiny value model (undefined, null, boolean, number,
 * string, object, array, array buffer, typed array, error, promise).  Asynchronous work
 * runs synchronously when queued.  Values are never freed: a test process is short.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../machinig-sim_b200/node/napi_min.h"
#include "fake_napi.h"

static struct napi_value__* alloc_value(fk_kind k) {
  struct napi_value__* v = (struct napi_value__*)calloc(1, sizeof(struct napi_value__));
  v->k = k;
  return v;
}

napi_value fk_undefined(void) { return alloc_value(FK_UNDEF); }
napi_value fk_null(void) { return alloc_value(FK_NULL); }
napi_value fk_bool(int b) {
  napi_value v = alloc_value(FK_BOOL);
  v->b = b;
  return v;
}
napi_value fk_num(double d) {
  napi_value v = alloc_value(FK_NUM);
  v->num = d;
  return v;
}
napi_value fk_str(const char* s) {
  napi_value v = alloc_value(FK_STR);
  v->s = strdup(s);
  return v;
}
napi_value fk_obj(void) { return alloc_value(FK_OBJ); }
napi_value fk_arr(void) { return alloc_value(FK_ARR); }

void fk_set(napi_value o, const char* key, napi_value v) {
  for (int i = 0; i < o->nprops; i++)
    if (strcmp(o->keys[i], key) == 0) {
      o->vals[i] = v;
      return;
    }
  if (o->nprops < FK_MAX_PROPS) {
    o->keys[o->nprops] = strdup(key);
    o->vals[o->nprops++] = v;
  }
}

napi_value fk_get(napi_value o, const char* key) {
  if (!o || (o->k != FK_OBJ && o->k != FK_ERR && o->k != FK_PROMISE)) return NULL;
  for (int i = 0; i < o->nprops; i++)
    if (strcmp(o->keys[i], key) == 0) return o->vals[i];
  return NULL;
}

void fk_push(napi_value a, napi_value v) {
  a->elems = (napi_value*)realloc(a->elems, sizeof(napi_value) * (size_t)(a->len + 1));
  a->elems[a->len++] = v;
}

/* ---- the runtime ---- */
struct napi_env__ g_env;

napi_status napi_get_cb_info(napi_env env, napi_callback_info cbinfo, size_t* argc,
                             napi_value* argv, napi_value* this_arg, void** data) {
  (void)env;
  (void)this_arg;
  (void)data;
  size_t n = *argc < cbinfo->argc ? *argc : cbinfo->argc;
  for (size_t i = 0; i < *argc; i++) argv[i] = i < n ? cbinfo->argv[i] : fk_undefined();
  *argc = cbinfo->argc;
  return napi_ok;
}

napi_status napi_typeof(napi_env env, napi_value v, napi_valuetype* r) {
  (void)env;
  if (!v) return napi_invalid_arg;
  switch (v->k) {
    case FK_UNDEF: *r = napi_undefined; break;
    case FK_NULL: *r = napi_null; break;
    case FK_BOOL: *r = napi_boolean; break;
    case FK_NUM: *r = napi_number; break;
    case FK_STR: *r = napi_string; break;
    default: *r = napi_object; break;
  }
  return napi_ok;
}

napi_status napi_get_named_property(napi_env env, napi_value o, const char* k, napi_value* r) {
  (void)env;
  napi_value v = fk_get(o, k);
  *r = v ? v : fk_undefined();
  return o && (o->k == FK_OBJ || o->k == FK_ERR) ? napi_ok : napi_object_expected;
}

napi_status napi_has_named_property(napi_env env, napi_value o, const char* k, bool* r) {
  (void)env;
  *r = fk_get(o, k) != NULL;
  return napi_ok;
}

napi_status napi_get_value_double(napi_env env, napi_value v, double* r) {
  (void)env;
  if (!v || v->k != FK_NUM) return napi_number_expected;
  *r = v->num;
  return napi_ok;
}

napi_status napi_get_value_bool(napi_env env, napi_value v, bool* r) {
  (void)env;
  if (!v || v->k != FK_BOOL) return napi_boolean_expected;
  *r = v->b != 0;
  return napi_ok;
}

napi_status napi_get_value_string_utf8(napi_env env, napi_value v, char* buf, size_t n,
                                       size_t* r) {
  (void)env;
  if (!v || v->k != FK_STR) return napi_string_expected;
  size_t len = strlen(v->s);
  if (buf && n) {
    size_t c = len < n - 1 ? len : n - 1;
    memcpy(buf, v->s, c);
    buf[c] = 0;
    len = c;
  }
  if (r) *r = len;
  return napi_ok;
}

napi_status napi_is_array(napi_env env, napi_value v, bool* r) {
  (void)env;
  *r = v && v->k == FK_ARR;
  return napi_ok;
}

napi_status napi_get_array_length(napi_env env, napi_value v, uint32_t* r) {
  (void)env;
  if (!v || v->k != FK_ARR) return napi_array_expected;
  *r = (uint32_t)v->len;
  return napi_ok;
}

napi_status napi_get_element(napi_env env, napi_value v, uint32_t i, napi_value* r) {
  (void)env;
  if (!v || v->k != FK_ARR) return napi_array_expected;
  *r = (int)i < v->len ? v->elems[i] : fk_undefined();
  return napi_ok;
}

napi_status napi_create_object(napi_env env, napi_value* r) {
  (void)env;
  *r = fk_obj();
  return napi_ok;
}

napi_status napi_create_array_with_length(napi_env env, size_t n, napi_value* r) {
  (void)env;
  *r = fk_arr();
  for (size_t i = 0; i < n; i++) fk_push(*r, fk_undefined());
  return napi_ok;
}

napi_status napi_set_element(napi_env env, napi_value a, uint32_t i, napi_value v) {
  (void)env;
  if (!a || a->k != FK_ARR) return napi_array_expected;
  while (a->len <= (int)i) fk_push(a, fk_undefined());
  a->elems[i] = v;
  return napi_ok;
}

napi_status napi_set_named_property(napi_env env, napi_value o, const char* k, napi_value v) {
  (void)env;
  fk_set(o, k, v);
  return napi_ok;
}

napi_status napi_create_double(napi_env env, double d, napi_value* r) {
  (void)env;
  *r = fk_num(d);
  return napi_ok;
}

napi_status napi_get_boolean(napi_env env, bool b, napi_value* r) {
  (void)env;
  *r = fk_bool(b);
  return napi_ok;
}

napi_status napi_get_undefined(napi_env env, napi_value* r) {
  (void)env;
  *r = fk_undefined();
  return napi_ok;
}

napi_status napi_create_string_utf8(napi_env env, const char* s, size_t len, napi_value* r) {
  (void)env;
  if (len == (size_t)-1) {
    *r = fk_str(s);
  } else {
    char* c = (char*)calloc(len + 1, 1);
    memcpy(c, s, len);
    *r = fk_str(c);
  }
  return napi_ok;
}

napi_status napi_create_error(napi_env env, napi_value code, napi_value msg, napi_value* r) {
  (void)env;
  *r = alloc_value(FK_ERR);
  if (code) fk_set(*r, "code", code);
  fk_set(*r, "message", msg);
  return napi_ok;
}

napi_status napi_throw_error(napi_env env, const char* code, const char* msg) {
  napi_value e;
  napi_create_error(env, code ? fk_str(code) : NULL, fk_str(msg ? msg : ""), &e);
  env->exception = e;
  return napi_ok;
}

napi_status napi_define_properties(napi_env env, napi_value o, size_t n,
                                   const napi_property_descriptor* p) {
  (void)env;
  for (size_t i = 0; i < n; i++) {
    napi_value f = alloc_value(FK_FUNC);
    f->fn = p[i].method;
    fk_set(o, p[i].utf8name, f);
  }
  return napi_ok;
}

napi_status napi_create_promise(napi_env env, napi_deferred* d, napi_value* promise) {
  (void)env;
  *d = (napi_deferred)calloc(1, sizeof(struct napi_deferred__));
  *promise = alloc_value(FK_PROMISE);
  (*d)->promise = *promise;
  return napi_ok;
}

napi_status napi_resolve_deferred(napi_env env, napi_deferred d, napi_value v) {
  (void)env;
  d->promise->b = 1;
  fk_set(d->promise, "value", v);
  d->promise->k = FK_PROMISE;
  return napi_ok;
}

napi_status napi_reject_deferred(napi_env env, napi_deferred d, napi_value v) {
  (void)env;
  d->promise->b = 2;
  fk_set(d->promise, "value", v);
  return napi_ok;
}

napi_status napi_create_async_work(napi_env env, napi_value res, napi_value name,
                                   napi_async_execute_callback exec,
                                   napi_async_complete_callback done, void* data,
                                   napi_async_work* r) {
  (void)env;
  (void)res;
  (void)name;
  *r = (napi_async_work)calloc(1, sizeof(struct napi_async_work__));
  (*r)->exec = exec;
  (*r)->done = done;
  (*r)->data = data;
  return napi_ok;
}

napi_status napi_queue_async_work(napi_env env, napi_async_work w) {
  w->exec(env, w->data);
  w->done(env, napi_ok, w->data);
  return napi_ok;
}

napi_status napi_delete_async_work(napi_env env, napi_async_work w) {
  (void)env;
  (void)w;
  return napi_ok;
}

napi_status napi_create_arraybuffer(napi_env env, size_t bytes, void** data, napi_value* r) {
  (void)env;
  *r = alloc_value(FK_AB);
  (*r)->data = calloc(bytes ? bytes : 1, 1);
  (*r)->bytes = bytes;
  if (data) *data = (*r)->data;
  return napi_ok;
}

napi_status napi_create_typedarray(napi_env env, napi_typedarray_type t, size_t n,
                                   napi_value ab, size_t off, napi_value* r) {
  (void)env;
  (void)t;
  *r = alloc_value(FK_TA);
  (*r)->data = (char*)ab->data + off;
  (*r)->len = (int)n;
  return napi_ok;
}

napi_value fk_call(napi_value exports, const char* name, int argc, napi_value* argv) {
  napi_value f = fk_get(exports, name);
  struct napi_callback_info__ info = {(size_t)argc, argv};
  g_env.exception = NULL;
  return f->fn(&g_env, &info);
}
