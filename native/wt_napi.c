/*
 * wt_napi.c — Node-API addon exposing libwt.so to the reference's TypeScript host.
 *
 * Implements the solver surface of src/backend/types.ts (LbmSolver / SolverFactory, lines 7-18,
 * and the compute half of Backend, lines 24-53) on the C ABI of include/wt.h. JS values are read
 * and built here; the rest (parameter mapping, the stepAndSample job, the SolverStats fields, the
 * voxelize argument packing, the export stride) is wt_addon.c, which tests/napi_sequence.c drives
 * without a JavaScript runtime. Built by binding.gyp (node-gyp) where Node's headers exist.
 *
 * Typed arrays are borrowed for the call only (libwt copies what it keeps). Handles are napi
 * externals whose finalizer calls wt_destroy; destroy() releases the handle at once. Calls on one
 * handle must not overlap: the TS adapter (native/cuda.ts) chains them per handle.
 */
#include <node_api.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wt_addon.h"

#define NAPI_CALL(env, expr)                                   \
  do {                                                         \
    if ((expr) != napi_ok) {                                   \
      napi_throw_error((env), NULL, "wt_napi: " #expr);        \
      return NULL;                                             \
    }                                                          \
  } while (0)

/* ---- handles ---------------------------------------------------------------------------------- */
typedef struct handle {
  wt_solver* s;
  wt_dims dims;
} handle;

static void finalize_handle(napi_env env, void* data, void* hint) {
  (void)env;
  (void)hint;
  handle* h = (handle*)data;
  if (h->s) wt_destroy(h->s);
  free(h);
}

static handle* get_handle(napi_env env, napi_value v) {
  void* p = NULL;
  if (napi_get_value_external(env, v, &p) != napi_ok || p == NULL || ((handle*)p)->s == NULL) {
    napi_throw_error(env, NULL, "wt_napi: not a live solver handle");
    return NULL;
  }
  return (handle*)p;
}

static napi_value throw_wt(napi_env env, const wt_solver* s, int rc) {
  char code[16];
  snprintf(code, sizeof code, "%d", rc);
  const char* m = wt_last_error(s);
  napi_throw_error(env, code, (m && m[0]) ? m : wt_error_string(rc));
  return NULL;
}

/* ---- JS value helpers ------------------------------------------------------------------------- */
static double get_num(napi_env env, napi_value obj, const char* key, double absent) {
  bool has = false;
  napi_value v;
  napi_valuetype t;
  double d = absent;
  if (napi_has_named_property(env, obj, key, &has) != napi_ok || !has) return absent;
  if (napi_get_named_property(env, obj, key, &v) != napi_ok || napi_typeof(env, v, &t) != napi_ok) return absent;
  if (t == napi_number) napi_get_value_double(env, v, &d);
  else if (t == napi_boolean) {
    bool b = false;
    napi_get_value_bool(env, v, &b);
    d = b ? 1.0 : 0.0;
  }
  return d;
}

/* copies the string property `key` into buf (NULL when absent or not a string) */
static const char* get_str(napi_env env, napi_value obj, const char* key, char* buf, size_t cap) {
  bool has = false;
  napi_value v;
  napi_valuetype t;
  size_t len = 0;
  if (napi_has_named_property(env, obj, key, &has) != napi_ok || !has) return NULL;
  if (napi_get_named_property(env, obj, key, &v) != napi_ok || napi_typeof(env, v, &t) != napi_ok) return NULL;
  if (t != napi_string || napi_get_value_string_utf8(env, v, buf, cap, &len) != napi_ok) return NULL;
  return buf;
}

static int get_typed(napi_env env, napi_value v, napi_typedarray_type want, void** data, size_t* len) {
  napi_typedarray_type t;
  if (napi_get_typedarray_info(env, v, &t, len, data, NULL, NULL) != napi_ok || t != want) return 0;
  return 1;
}

static void set_num(napi_env env, napi_value o, const char* k, double v) {
  napi_value x;
  napi_create_double(env, v, &x);
  napi_set_named_property(env, o, k, x);
}

static napi_value stats_object(napi_env env, const wt_stats* st) {
  napi_value o, b;
  wta_field f[WTA_STATS_FIELDS];
  napi_create_object(env, &o);
  wta_stats_fields(st, f);
  for (int k = 0; k < WTA_STATS_FIELDS; k++) {
    if (strcmp(f[k].name, "unstable") == 0) {
      napi_get_boolean(env, f[k].value != 0.0, &b);
      napi_set_named_property(env, o, f[k].name, b);
    } else {
      set_num(env, o, f[k].name, f[k].value);
    }
  }
  return o;
}

/* SolverParams object -> wt_params (wta_make_params) */
static int read_params(napi_env env, napi_value obj, wt_params* out) {
  char g[16], sd[16], pr[16], co[16];
  wta_solver_params in;
  const char* why = NULL;
  wta_params_init(&in);
  in.u = get_num(env, obj, "u", NAN);
  in.nu = get_num(env, obj, "nu", NAN);
  in.cs = get_num(env, obj, "cs", 0.0);
  in.sponge_nu = get_num(env, obj, "spongeNu", 0.0);
  in.sponge_start = get_num(env, obj, "spongeStart", 1.0);
  in.sponge_in = get_num(env, obj, "spongeIn", NAN);
  in.tau_wall = get_num(env, obj, "tauWall", NAN);
  in.ema_alpha = get_num(env, obj, "emaAlpha", 0.0);
  in.ground = get_str(env, obj, "ground", g, sizeof g);
  in.sides = get_str(env, obj, "sides", sd, sizeof sd);
  in.precision = get_str(env, obj, "precision", pr, sizeof pr);
  in.collision = get_str(env, obj, "collision", co, sizeof co);
  in.interp = (int32_t)get_num(env, obj, "interp", -1.0);
  if (wta_make_params(&in, out, &why) != WT_OK) {
    char m[96];
    snprintf(m, sizeof m, "wt_napi: bad SolverParams field '%s'", why ? why : "?");
    napi_throw_type_error(env, NULL, m);
    return 0;
  }
  return 1;
}

/* ---- SolverFactory / LbmSolver ---------------------------------------------------------------- */
/* create(dims {nx, ny, nz}, SolverParams) -> handle */
static napi_value js_create(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2], out;
  wt_params p;
  handle* h;
  wt_solver* s = NULL;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  wt_dims d = {(int32_t)get_num(env, argv[0], "nx", 0), (int32_t)get_num(env, argv[0], "ny", 0),
               (int32_t)get_num(env, argv[0], "nz", 1)};
  if (!read_params(env, argv[1], &p)) return NULL;
  int rc = wt_create(&d, &p, &s);
  if (rc != WT_OK) return throw_wt(env, NULL, rc);
  h = (handle*)calloc(1, sizeof *h);
  h->s = s;
  h->dims = d;
  NAPI_CALL(env, napi_create_external(env, h, finalize_handle, NULL, &out));
  return out;
}

/* destroy(handle): releases the device memory now (the finalizer then has nothing left to do) */
static napi_value js_destroy(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  void* p = NULL;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (napi_get_value_external(env, argv[0], &p) == napi_ok && p) {
    handle* h = (handle*)p;
    wt_destroy(h->s);
    h->s = NULL;
  }
  return NULL;
}

/* uploadFlags(handle, Uint32Array) / uploadSdf(handle, Float32Array) */
static napi_value js_upload(napi_env env, napi_callback_info info, int sdf) {
  size_t argc = 2, len = 0;
  napi_value argv[2];
  void* data = NULL;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h) return NULL;
  if (!get_typed(env, argv[1], sdf ? napi_float32_array : napi_uint32_array, &data, &len)) {
    napi_throw_type_error(env, NULL, sdf ? "uploadSdf: Float32Array expected" : "uploadFlags: Uint32Array expected");
    return NULL;
  }
  int rc = sdf ? wt_upload_sdf(h->s, (const float*)data, (int64_t)len)
               : wt_upload_flags(h->s, (const uint32_t*)data, (int64_t)len);
  return rc == WT_OK ? NULL : throw_wt(env, h->s, rc);
}
static napi_value js_upload_flags(napi_env env, napi_callback_info info) { return js_upload(env, info, 0); }
static napi_value js_upload_sdf(napi_env env, napi_callback_info info) { return js_upload(env, info, 1); }

/* stepAndSample(handle, steps) -> Promise<SolverStats>, stepped on the libuv pool */
typedef struct step_work {
  napi_async_work work;
  napi_deferred deferred;
  wta_step_job job;
} step_work;

static void step_execute(napi_env env, void* data) {
  (void)env;
  wta_step_job_execute(&((step_work*)data)->job);
}

static void step_complete(napi_env env, napi_status status, void* data) {
  step_work* w = (step_work*)data;
  if (status != napi_ok || w->job.rc != WT_OK) {
    napi_value msg, err;
    napi_create_string_utf8(env, w->job.err[0] ? w->job.err : "stepAndSample failed", NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, NULL, msg, &err);
    napi_reject_deferred(env, w->deferred, err);
  } else {
    napi_resolve_deferred(env, w->deferred, stats_object(env, &w->job.st));
  }
  napi_delete_async_work(env, w->work);
  free(w);
}

static napi_value js_step_and_sample(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2], promise, name;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h) return NULL;
  step_work* w = (step_work*)calloc(1, sizeof *w);
  w->job.s = h->s;
  if (napi_get_value_int32(env, argv[1], &w->job.steps) != napi_ok || w->job.steps < 0) {
    free(w);
    napi_throw_range_error(env, NULL, "stepAndSample: steps must be a non-negative integer");
    return NULL;
  }
  NAPI_CALL(env, napi_create_promise(env, &w->deferred, &promise));
  NAPI_CALL(env, napi_create_string_utf8(env, "wt_step_and_sample", NAPI_AUTO_LENGTH, &name));
  NAPI_CALL(env, napi_create_async_work(env, NULL, name, step_execute, step_complete, w, &w->work));
  NAPI_CALL(env, napi_queue_async_work(env, w->work));
  return promise;
}

/* ---- Backend ---------------------------------------------------------------------------------- */
/* setParams(handle, SolverParams) — the TS side merges the Partial into its full copy first */
static napi_value js_set_params(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  wt_params p;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h || !read_params(env, argv[1], &p)) return NULL;
  int rc = wt_set_params(h->s, &p);
  return rc == WT_OK ? NULL : throw_wt(env, h->s, rc);
}

static napi_value js_simple(napi_env env, napi_callback_info info, int (*fn)(wt_solver*)) {
  size_t argc = 1;
  napi_value argv[1];
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h) return NULL;
  int rc = fn(h->s);
  return rc == WT_OK ? NULL : throw_wt(env, h->s, rc);
}
static napi_value js_reset(napi_env env, napi_callback_info info) { return js_simple(env, info, wt_reset); }
static napi_value js_clear_stats(napi_env env, napi_callback_info info) { return js_simple(env, info, wt_clear_stats); }

/* voxelize(handle, Float32Array positions | null, Uint32Array indices | null, Float64Array(16)
 * matrix, Float64Array wheels (8 per wheel)) -> VoxelInfo */
static napi_value js_voxelize(napi_env env, napi_callback_info info) {
  size_t argc = 5, npos = 0, nidx = 0, nm = 0, nw = 0;
  napi_value argv[5], o, arr, x;
  napi_valuetype t;
  void *pos = NULL, *idx = NULL, *m = NULL, *wh = NULL;
  wt_voxel_info vi;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h) return NULL;
  NAPI_CALL(env, napi_typeof(env, argv[1], &t));
  if (t != napi_null && (!get_typed(env, argv[1], napi_float32_array, &pos, &npos) ||
                         !get_typed(env, argv[2], napi_uint32_array, &idx, &nidx))) {
    napi_throw_type_error(env, NULL, "voxelize: Float32Array positions and Uint32Array indices expected");
    return NULL;
  }
  if (!get_typed(env, argv[3], napi_float64_array, &m, &nm) || nm != 16 ||
      !get_typed(env, argv[4], napi_float64_array, &wh, &nw)) {
    napi_throw_type_error(env, NULL, "voxelize: Float64Array(16) matrix and Float64Array wheels expected");
    return NULL;
  }
  int rc = wta_voxelize(h->s, (const float*)pos, npos, (const uint32_t*)idx, nidx, (const double*)m,
                        (const double*)wh, nw, &vi);
  if (rc != WT_OK) return throw_wt(env, h->s, rc);
  napi_create_object(env, &o);
  set_num(env, o, "frontal", vi.frontal);
  set_num(env, o, "solidCells", vi.solid_cells);
  napi_create_array_with_length(env, 3, &arr);
  for (uint32_t a = 0; a < 3; a++) {
    napi_create_int32(env, vi.min[a], &x);
    napi_set_element(env, arr, a, x);
  }
  napi_set_named_property(env, o, "min", arr);
  napi_create_array_with_length(env, 3, &arr);
  for (uint32_t a = 0; a < 3; a++) {
    napi_create_int32(env, vi.max[a], &x);
    napi_set_element(env, arr, a, x);
  }
  napi_set_named_property(env, o, "max", arr);
  return o;
}

/* readVelocity(handle, Float32Array(4 n)): the velocity texture of the last sample */
static napi_value js_read_velocity(napi_env env, napi_callback_info info) {
  size_t argc = 2, len = 0;
  napi_value argv[2];
  void* data = NULL;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h) return NULL;
  if (!get_typed(env, argv[1], napi_float32_array, &data, &len)) {
    napi_throw_type_error(env, NULL, "readVelocity: Float32Array expected");
    return NULL;
  }
  int rc = wt_read_velocity(h->s, (float*)data, (int64_t)(len / 4));
  return rc == WT_OK ? NULL : throw_wt(env, h->s, rc);
}

/* exportFields(handle, maxPoints) -> {stride, dims: [px, py, pz], vel, mean, vort} (FieldExport,
 * src/solver/types.ts:45-54), sub-sampled as Backend.exportFields does */
static napi_value js_export_fields(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2], o, ab[3], ta[3], dims, x;
  double maxp = 0;
  void* buf[3];
  static const char* const names[3] = {"vel", "mean", "vort"};
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  handle* h = get_handle(env, argv[0]);
  if (!h) return NULL;
  NAPI_CALL(env, napi_get_value_double(env, argv[1], &maxp));
  const int32_t stride = wta_export_stride(&h->dims, maxp > 1 ? maxp : 1);
  const int64_t pts = wta_export_points(&h->dims, stride);
  for (int k = 0; k < 3; k++) {
    NAPI_CALL(env, napi_create_arraybuffer(env, (size_t)pts * 16, &buf[k], &ab[k]));
    NAPI_CALL(env, napi_create_typedarray(env, napi_float32_array, (size_t)pts * 4, ab[k], 0, &ta[k]));
  }
  int rc = wt_export_fields(h->s, stride, (float*)buf[0], (float*)buf[1], (float*)buf[2], pts);
  if (rc != WT_OK) return throw_wt(env, h->s, rc);
  napi_create_object(env, &o);
  set_num(env, o, "stride", stride);
  napi_create_array_with_length(env, 3, &dims);
  const int32_t pd[3] = {(h->dims.nx + stride - 1) / stride, (h->dims.ny + stride - 1) / stride,
                         (h->dims.nz + stride - 1) / stride};
  for (uint32_t a = 0; a < 3; a++) {
    napi_create_int32(env, pd[a], &x);
    napi_set_element(env, dims, a, x);
  }
  napi_set_named_property(env, o, "dims", dims);
  for (int k = 0; k < 3; k++) napi_set_named_property(env, o, names[k], ta[k]);
  return o;
}

/* fits(dims, precision) -> boolean (Backend.fits) */
static napi_value js_fits(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2], out;
  char pr[16];
  int64_t bytes = 0;
  int32_t ok = 0;
  NAPI_CALL(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  wt_dims d = {(int32_t)get_num(env, argv[0], "nx", 0), (int32_t)get_num(env, argv[0], "ny", 0),
               (int32_t)get_num(env, argv[0], "nz", 1)};
  const char* p = argc > 1 ? get_str(env, argv[1], "precision", pr, sizeof pr) : NULL;
  const int prec = (p && strcmp(p, "f16") == 0) ? WT_PREC_F16 : WT_PREC_F32;
  int rc = wt_fits(&d, prec, &bytes, &ok);
  if (rc != WT_OK) return throw_wt(env, NULL, rc);
  NAPI_CALL(env, napi_get_boolean(env, ok != 0, &out));
  return out;
}

NAPI_MODULE_INIT() {
  napi_property_descriptor d[] = {
      {"create", NULL, js_create, NULL, NULL, NULL, napi_default, NULL},
      {"destroy", NULL, js_destroy, NULL, NULL, NULL, napi_default, NULL},
      {"uploadFlags", NULL, js_upload_flags, NULL, NULL, NULL, napi_default, NULL},
      {"uploadSdf", NULL, js_upload_sdf, NULL, NULL, NULL, napi_default, NULL},
      {"stepAndSample", NULL, js_step_and_sample, NULL, NULL, NULL, napi_default, NULL},
      {"setParams", NULL, js_set_params, NULL, NULL, NULL, napi_default, NULL},
      {"reset", NULL, js_reset, NULL, NULL, NULL, napi_default, NULL},
      {"clearStats", NULL, js_clear_stats, NULL, NULL, NULL, napi_default, NULL},
      {"voxelize", NULL, js_voxelize, NULL, NULL, NULL, napi_default, NULL},
      {"readVelocity", NULL, js_read_velocity, NULL, NULL, NULL, napi_default, NULL},
      {"exportFields", NULL, js_export_fields, NULL, NULL, NULL, napi_default, NULL},
      {"fits", NULL, js_fits, NULL, NULL, NULL, napi_default, NULL},
  };
  if (napi_define_properties(env, exports, sizeof d / sizeof d[0], d) != napi_ok) return NULL;
  return exports;
}
