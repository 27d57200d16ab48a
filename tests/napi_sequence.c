/*
 * napi_sequence.c — runs the N-API addon's call sequence (native/wt_napi.c) without a JavaScript
 * runtime, through the addon's own C half (native/wt_addon.c) and libwt.so.
 *
 *   napi_sequence params KEY=VALUE ...
 *       SolverParams -> wt_params as the addon maps them; prints the mapped struct as one JSON line
 *   napi_sequence run DIR NX NY NZ STEPS CHUNKS KEY=VALUE ...
 *       create -> uploadFlags (DIR/flags.u32) -> uploadSdf (DIR/sdf.f32) -> CHUNKS x
 *       stepAndSample(STEPS) -> readVelocity -> destroy; writes DIR/stats.f64 (the SolverStats
 *       fields of every chunk, WTA_STATS_FIELDS doubles each) and DIR/velocity.f32 (4 per cell)
 *
 * KEY is a SolverParams field name (u, nu, cs, spongeNu, spongeStart, spongeIn, tauWall, emaAlpha,
 * ground, sides, precision, collision, interp). Exit code 0 on success, else the WT_E_* code's
 * absolute value (or 100 for a usage / file error), with the message on stderr.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wt_addon.h"

static void parse_param(wta_solver_params* p, const char* kv) {
  char key[32];
  const char* eq = strchr(kv, '=');
  if (!eq || (size_t)(eq - kv) >= sizeof key) return;
  memcpy(key, kv, (size_t)(eq - kv));
  key[eq - kv] = '\0';
  const char* v = eq + 1;
  if (!strcmp(key, "u")) p->u = atof(v);
  else if (!strcmp(key, "nu")) p->nu = atof(v);
  else if (!strcmp(key, "cs")) p->cs = atof(v);
  else if (!strcmp(key, "spongeNu")) p->sponge_nu = atof(v);
  else if (!strcmp(key, "spongeStart")) p->sponge_start = atof(v);
  else if (!strcmp(key, "spongeIn")) p->sponge_in = atof(v);
  else if (!strcmp(key, "tauWall")) p->tau_wall = atof(v);
  else if (!strcmp(key, "emaAlpha")) p->ema_alpha = atof(v);
  else if (!strcmp(key, "ground")) p->ground = v;
  else if (!strcmp(key, "sides")) p->sides = v;
  else if (!strcmp(key, "precision")) p->precision = v;
  else if (!strcmp(key, "collision")) p->collision = v;
  else if (!strcmp(key, "interp")) p->interp = (!strcmp(v, "false") || !strcmp(v, "0")) ? 0 : 1;
}

static int read_file(const char* dir, const char* name, void* dst, size_t bytes) {
  char path[1024];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* f = fopen(path, "rb");
  if (!f) return 0;
  const size_t got = fread(dst, 1, bytes, f);
  fclose(f);
  return got == bytes;
}

static int write_file(const char* dir, const char* name, const void* src, size_t bytes) {
  char path[1024];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* f = fopen(path, "wb");
  if (!f) return 0;
  const size_t put = fwrite(src, 1, bytes, f);
  fclose(f);
  return put == bytes;
}

static int fail(int rc, const wt_solver* s, const char* what) {
  const char* m = wt_last_error(s);
  fprintf(stderr, "%s: %s (%d)\n", what, (m && m[0]) ? m : wt_error_string(rc), rc);
  return rc < 0 ? -rc : 100;
}

int main(int argc, char** argv) {
  wta_solver_params in;
  wt_params p;
  const char* why = NULL;
  wta_params_init(&in);
  if (argc >= 2 && !strcmp(argv[1], "params")) {
    for (int k = 2; k < argc; k++) parse_param(&in, argv[k]);
    if (wta_make_params(&in, &p, &why) != WT_OK) {
      printf("{\"error\": \"%s\"}\n", why ? why : "?");
      return 0;
    }
    printf("{\"u\": %.17g, \"nu\": %.17g, \"cs\": %.17g, \"sponge_nu\": %.17g, \"sponge_start\": %.17g, "
           "\"sponge_in\": %.17g, \"tau_wall\": %.17g, \"ema_alpha\": %.17g, \"ground\": %d, \"sides\": %d, "
           "\"precision\": %d, \"interp\": %d, \"collision\": %d, \"init_mode\": %d}\n",
           p.u, p.nu, p.cs, p.sponge_nu, p.sponge_start, p.sponge_in, p.tau_wall, p.ema_alpha, p.ground, p.sides,
           p.precision, p.interp, p.collision, p.init_mode);
    return 0;
  }
  if (argc < 8 || strcmp(argv[1], "run") != 0) {
    fprintf(stderr, "usage: napi_sequence params KEY=VALUE ... | run DIR NX NY NZ STEPS CHUNKS KEY=VALUE ...\n");
    return 100;
  }
  const char* dir = argv[2];
  const wt_dims d = {atoi(argv[3]), atoi(argv[4]), atoi(argv[5])};
  const int32_t steps = atoi(argv[6]);
  const int chunks = atoi(argv[7]);
  for (int k = 8; k < argc; k++) parse_param(&in, argv[k]);
  if (wta_make_params(&in, &p, &why) != WT_OK) {
    fprintf(stderr, "bad SolverParams field %s\n", why ? why : "?");
    return 100;
  }
  const size_t n = (size_t)d.nx * (size_t)d.ny * (size_t)d.nz;
  uint32_t* flags = (uint32_t*)malloc(n * 4);
  float* sdf = (float*)malloc(n * 4);
  float* vel = (float*)malloc(n * 16);
  double* stats = (double*)calloc((size_t)chunks * WTA_STATS_FIELDS, sizeof(double));
  if (!flags || !sdf || !vel || !stats || !read_file(dir, "flags.u32", flags, n * 4) ||
      !read_file(dir, "sdf.f32", sdf, n * 4)) {
    fprintf(stderr, "cannot read the geometry from %s\n", dir);
    return 100;
  }
  /* SolverFactory(dims, params) */
  wt_solver* s = NULL;
  int rc = wt_create(&d, &p, &s);
  if (rc != WT_OK) return fail(rc, NULL, "create");
  /* uploadFlags / uploadSdf */
  if ((rc = wt_upload_flags(s, flags, (int64_t)n)) != WT_OK) return fail(rc, s, "uploadFlags");
  if ((rc = wt_upload_sdf(s, sdf, (int64_t)n)) != WT_OK) return fail(rc, s, "uploadSdf");
  /* stepAndSample, each call as the job the addon queues on the libuv pool */
  for (int c = 0; c < chunks; c++) {
    wta_step_job job;
    wta_field f[WTA_STATS_FIELDS];
    memset(&job, 0, sizeof job);
    job.s = s;
    job.steps = steps;
    wta_step_job_execute(&job);
    if (job.rc != WT_OK) {
      fprintf(stderr, "stepAndSample: %s\n", job.err);
      return -job.rc;
    }
    wta_stats_fields(&job.st, f);
    for (int k = 0; k < WTA_STATS_FIELDS; k++) stats[(size_t)c * WTA_STATS_FIELDS + k] = f[k].value;
  }
  /* readVelocity */
  if ((rc = wt_read_velocity(s, vel, (int64_t)n)) != WT_OK) return fail(rc, s, "readVelocity");
  /* destroy */
  wt_destroy(s);
  if (!write_file(dir, "stats.f64", stats, (size_t)chunks * WTA_STATS_FIELDS * sizeof(double)) ||
      !write_file(dir, "velocity.f32", vel, n * 16)) {
    fprintf(stderr, "cannot write the results to %s\n", dir);
    return 100;
  }
  free(flags);
  free(sdf);
  free(vel);
  free(stats);
  return 0;
}
