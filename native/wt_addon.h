/*
 * wt_addon.h — the Node-independent half of the N-API addon (native/wt_napi.c).
 *
 * The addon turns the reference's TypeScript solver calls into calls of the C ABI (include/wt.h).
 * Everything it does apart from reading and building JS values lives here, in plain C, so that a
 * C program can run the addon's exact call sequence without a JavaScript runtime:
 *
 *   SolverFactory (src/backend/types.ts:18) .... wta_make_params + wt_create
 *   LbmSolver.uploadFlags / uploadSdf (:11-13) .. wt_upload_flags / wt_upload_sdf
 *   LbmSolver.stepAndSample (:14) ............... wta_step_job_execute (on the libuv pool) and
 *                                                 wta_stats_fields (the SolverStats object)
 *   Backend.voxelize (:36) ...................... wta_voxelize
 *   Backend.exportFields (:51) .................. wta_export_stride + wt_export_fields
 *   LbmSolver.destroy (:15) ..................... wt_destroy (the handle's finalizer)
 */
#ifndef WT_ADDON_H
#define WT_ADDON_H

#include <stddef.h>
#include <stdint.h>

#include "wt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* SolverParams (src/solver/types.ts:3-29) as the JS object holds it. Optional fields the object
 * does not have are NaN (numbers), NULL (strings) or -1 (interp); the reference's defaults then
 * apply: spongeIn 0, tauWall 0.5, precision 'f32', interp true, collision 'regularized'. */
typedef struct wta_solver_params {
  double u, nu, cs;
  double sponge_nu, sponge_start;
  double sponge_in;      /* NaN: absent */
  double tau_wall;       /* NaN: absent */
  double ema_alpha;
  const char* ground;    /* 'freeslip' | 'noslip' | 'moving' */
  const char* sides;     /* 'freeslip' | 'periodic'; NULL: 'freeslip' */
  const char* precision; /* 'f32' | 'f16' (and the extension 'f64'); NULL: 'f32' */
  const char* collision; /* 'regularized' | 'bgk'; NULL: 'regularized' */
  int32_t interp;        /* 1 true, 0 false, -1 absent */
} wta_solver_params;

/* Fills every field of `in` with "absent" (numbers 0 where the reference requires them). */
void wta_params_init(wta_solver_params* in);

/* SolverParams -> wt_params. WT_OK, or WT_E_INVALID with *why naming the bad field. */
int wta_make_params(const wta_solver_params* in, wt_params* out, const char** why);

/* One stepAndSample call: queued by the addon on the libuv pool (napi_create_async_work), executed
 * off the JS thread, and resolved or rejected on it. `err` holds wt_last_error on failure. */
typedef struct wta_step_job {
  wt_solver* s;
  int32_t steps;
  int rc;
  wt_stats st;
  char err[256];
} wta_step_job;
void wta_step_job_execute(wta_step_job* job);

/* The SolverStats object (src/solver/types.ts:31-42) the Promise resolves to, in the order the
 * addon sets its properties: fx, fy, fz, maxU, rhoRef, unstable (0 / 1, a boolean in JS), step,
 * and the extension mass (FP64 sum of the fluid densities). */
#define WTA_STATS_FIELDS 8
typedef struct wta_field {
  const char* name;
  double value;
} wta_field;
void wta_stats_fields(const wt_stats* st, wta_field out[WTA_STATS_FIELDS]);

/* Backend.voxelize(mesh, matrix, wheels): positions (3 floats per vertex) and indices (3 per
 * triangle) of the mesh, the placement matrix as the JS numbers of placementMatrix
 * (src/voxelize/mesh.ts:354-379, column-major; rounded to f32 here as the reference writes it into
 * a Float32Array uniform) and the WheelDefs packed 8 doubles each (c xyz, axis xyz, r, hw). A
 * NULL mesh (npos == 0) clears the geometry. */
int wta_voxelize(wt_solver* s, const float* pos, size_t npos_floats, const uint32_t* idx, size_t nidx,
                 const double* matrix16, const double* wheels8, size_t nwheel_doubles, wt_voxel_info* info);

/* Backend.exportFields(maxPoints) (src/backend/webgpu.ts:133-137): the stride
 * max(1, ceil(cbrt(n / maxPoints))) and the number of points wt_export_fields fills at it. */
int32_t wta_export_stride(const wt_dims* d, double max_points);
int64_t wta_export_points(const wt_dims* d, int32_t stride);

#ifdef __cplusplus
}
#endif

#endif /* WT_ADDON_H */
