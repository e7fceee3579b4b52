/* Value model of the test stand-in for the Node-API runtime (fake_napi.c). */
#ifndef MCS_FAKE_NAPI_H_
#define MCS_FAKE_NAPI_H_

#include "../../machinig-sim_b200/node/napi_min.h"

#define FK_MAX_PROPS 32

typedef enum {
  FK_UNDEF, FK_NULL, FK_BOOL, FK_NUM, FK_STR, FK_OBJ, FK_ARR, FK_FUNC, FK_AB, FK_TA, FK_ERR,
  FK_PROMISE
} fk_kind;

struct napi_value__ {
  fk_kind k;
  double num;
  int b; /* boolean; for a promise 0 pending, 1 resolved, 2 rejected */
  char* s;
  int nprops;
  char* keys[FK_MAX_PROPS];
  struct napi_value__* vals[FK_MAX_PROPS];
  int len;
  struct napi_value__** elems;
  void* data;
  size_t bytes;
  napi_callback fn;
};
struct napi_env__ {
  napi_value exception;
};
struct napi_callback_info__ {
  size_t argc;
  napi_value* argv;
};
struct napi_deferred__ {
  napi_value promise;
};
struct napi_async_work__ {
  napi_async_execute_callback exec;
  napi_async_complete_callback done;
  void* data;
};

extern struct napi_env__ g_env;

napi_value fk_undefined(void);
napi_value fk_null(void);
napi_value fk_bool(int b);
napi_value fk_num(double d);
napi_value fk_str(const char* s);
napi_value fk_obj(void);
napi_value fk_arr(void);
void fk_set(napi_value o, const char* key, napi_value v);
napi_value fk_get(napi_value o, const char* key);
void fk_push(napi_value a, napi_value v);
napi_value fk_call(napi_value exports, const char* name, int argc, napi_value* argv);

#endif
