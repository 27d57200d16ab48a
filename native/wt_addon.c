/* wt_addon.c — see wt_addon.h. Plain C99; links against libwt.so. */
#include "wt_addon.h"

#include <math.h>
#include <string.h>

void wta_params_init(wta_solver_params* in) {
  memset(in, 0, sizeof *in);
  in->sponge_start = 1.0;
  in->sponge_in = NAN;
  in->tau_wall = NAN;
  in->interp = -1;
}

static int pick(const char* v, const char* const* names, int count, int def, int* out) {
  if (v == NULL) {
    *out = def;
    return 1;
  }
  for (int k = 0; k < count; k++)
    if (strcmp(v, names[k]) == 0) {
      *out = k;
      return 1;
    }
  return 0;
}

int wta_make_params(const wta_solver_params* in, wt_params* out, const char** why) {
  static const char* const ground[] = {"freeslip", "noslip", "moving"};        /* WT_GROUND_* */
  static const char* const sides[] = {"freeslip", "periodic"};                 /* WT_SIDES_* */
  static const char* const precision[] = {"f32", "f16", "f64"};                /* WT_PREC_* */
  static const char* const collision[] = {"regularized", "bgk"};               /* WT_COLL_* */
  const char* bad = NULL;
  int g = 0, sd = 0, pr = 0, co = 0;
  memset(out, 0, sizeof *out);
  if (!pick(in->ground, ground, 3, WT_GROUND_FREESLIP, &g)) bad = "ground";
  else if (!pick(in->sides, sides, 2, WT_SIDES_FREESLIP, &sd)) bad = "sides";
  else if (!pick(in->precision, precision, 3, WT_PREC_F32, &pr)) bad = "precision";
  else if (!pick(in->collision, collision, 2, WT_COLL_REGULARIZED, &co)) bad = "collision";
  else if (!isfinite(in->u) || !isfinite(in->nu)) bad = "u / nu";
  if (bad) {
    if (why) *why = bad;
    return WT_E_INVALID;
  }
  out->u = in->u;
  out->nu = in->nu;
  out->cs = in->cs;
  out->sponge_nu = in->sponge_nu;
  out->sponge_start = in->sponge_start;
  out->sponge_in = isnan(in->sponge_in) ? 0.0 : in->sponge_in;
  out->tau_wall = isnan(in->tau_wall) ? 0.5 : in->tau_wall;
  out->ema_alpha = in->ema_alpha;
  out->init_noise = 1e-4;
  out->ground = g;
  out->sides = sd;
  out->precision = pr;
  out->interp = in->interp == 0 ? 0 : 1;
  out->collision = co;
  out->init_mode = WT_INIT_FREESTREAM; /* the reference's reset: the free-stream equilibrium */
  out->init_seed = 1;
  if (why) *why = NULL;
  return WT_OK;
}

void wta_step_job_execute(wta_step_job* job) {
  job->err[0] = '\0';
  job->rc = wt_step_and_sample(job->s, job->steps, &job->st);
  if (job->rc != WT_OK) {
    const char* m = wt_last_error(job->s);
    strncpy(job->err, m ? m : wt_error_string(job->rc), sizeof job->err - 1);
    job->err[sizeof job->err - 1] = '\0';
  }
}

void wta_stats_fields(const wt_stats* st, wta_field out[WTA_STATS_FIELDS]) {
  const wta_field f[WTA_STATS_FIELDS] = {
      {"fx", st->fx},         {"fy", st->fy},
      {"fz", st->fz},         {"maxU", st->max_u},
      {"rhoRef", st->rho_ref}, {"unstable", st->unstable ? 1.0 : 0.0},
      {"step", (double)st->step}, {"mass", st->mass},
  };
  memcpy(out, f, sizeof f);
}

int wta_voxelize(wt_solver* s, const float* pos, size_t npos_floats, const uint32_t* idx, size_t nidx,
                 const double* matrix16, const double* wheels8, size_t nwheel_doubles, wt_voxel_info* info) {
  float m[16];
  wt_wheel w[16];
  int32_t nw = (int32_t)(nwheel_doubles / 8);
  if (nw > 16) nw = 16;
  if (matrix16 == NULL || npos_floats % 3 != 0 || nidx % 3 != 0 || nwheel_doubles % 8 != 0) return WT_E_INVALID;
  for (int k = 0; k < 16; k++) m[k] = (float)matrix16[k];
  for (int32_t k = 0; k < nw; k++) {
    const double* src = wheels8 + 8 * (size_t)k;
    for (int a = 0; a < 3; a++) {
      w[k].c[a] = src[a];
      w[k].axis[a] = src[3 + a];
    }
    w[k].r = src[6];
    w[k].hw = src[7];
  }
  return wt_voxelize(s, pos, (int64_t)(npos_floats / 3), idx, (int64_t)(nidx / 3), m, nw > 0 ? w : NULL, nw, info);
}

int32_t wta_export_stride(const wt_dims* d, double max_points) {
  const double n = (double)d->nx * (double)d->ny * (double)d->nz;
  const double s = ceil(cbrt(n / max_points));
  return s > 1.0 ? (int32_t)s : 1;
}

int64_t wta_export_points(const wt_dims* d, int32_t stride) {
  const int64_t px = (d->nx + stride - 1) / stride, py = (d->ny + stride - 1) / stride,
                pz = (d->nz + stride - 1) / stride;
  return px * py * pz;
}
