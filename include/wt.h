/*
 * wt.h — C ABI of the B200 lattice Boltzmann wind-tunnel compute path.
 *
 * This is the drop-in boundary for the reference's compute path. Every entry point replaces one
 * method of the reference's solver / backend objects (TypeScript over WebGPU); the citation on
 * each line names the interface it stands in for (paths relative to the reference project).
 *
 *   LbmSolver / SolverFactory ............ src/backend/types.ts:7-18
 *   Backend (fits, voxelize, setParams…) . src/backend/types.ts:24-53
 *   SolverGPU (the WebGPU solver object) . src/solver/SolverGPU.ts:12-444
 *   VoxelizerGPU.voxelize ................ src/voxelize/VoxelizerGPU.ts:48-151
 *   particle tracers ..................... src/render/tracers.ts:3-106, RendererGPU.ts:505-527
 *
 * Conventions
 *   - Cell index everywhere: cell = x + nx * (y + ny * z). D2Q9 when nz == 1, D3Q19 otherwise.
 *   - Populations are structure-of-arrays: f[i * N + cell]. FP16 storage holds (f_i - w_i) as IEEE
 *     binary16, which is byte-for-byte the reference's packed pair layout (two cells per u32 word,
 *     low half = even cell).
 *   - Host pointers are borrowed for the duration of the call only (copied, never retained).
 *   - Device memory is owned by the handle and released by wt_destroy.
 *   - Every function returns WT_OK (0) or a negative WT_E_* code and stores a message retrievable
 *     with wt_last_error(); nothing aborts or throws across the ABI.
 *   - Calls on one handle must be serialised by the caller. Each handle owns one CUDA stream on the
 *     device that was current when it was created, so handles are independent of each other.
 */
#ifndef WT_H
#define WT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WT_ABI_VERSION 2

enum {
  WT_OK = 0,
  WT_E_INVALID = -1,     /* bad argument: null pointer, size mismatch, unsupported dims */
  WT_E_CUDA = -2,        /* CUDA runtime error (message holds cudaGetErrorString) */
  WT_E_OOM = -3,         /* device allocation failed */
  WT_E_STATE = -4,       /* call not valid in the handle's current state */
  WT_E_UNSUPPORTED = -5, /* feature not available for this precision / lattice */
  WT_E_NO_DEVICE = -6    /* no CUDA device visible */
};

enum { WT_GROUND_FREESLIP = 0, WT_GROUND_NOSLIP = 1, WT_GROUND_MOVING = 2 };
enum { WT_SIDES_FREESLIP = 0, WT_SIDES_PERIODIC = 1 };
enum { WT_PREC_F32 = 0, WT_PREC_F16 = 1, WT_PREC_F64 = 2 };
enum { WT_COLL_REGULARIZED = 0, WT_COLL_BGK = 1 };
enum { WT_INIT_FREESTREAM = 0, WT_INIT_REST_NOISE = 1 };

typedef struct wt_dims {
  int32_t nx, ny, nz;
} wt_dims;

/* SolverParams (src/solver/types.ts:3-29). Real-valued fields are doubles because the reference
 * holds them as JS numbers and rounds only the derived values to f32 when it packs the uniform. */
typedef struct wt_params {
  double u;            /* lattice inlet velocity (cells / step) */
  double nu;           /* molecular lattice viscosity */
  double cs;           /* Smagorinsky constant */
  double sponge_nu;    /* extra viscosity in the outlet sponge */
  double sponge_start; /* fraction of nx where the outlet sponge starts */
  double sponge_in;    /* width (fraction of nx) of the inlet absorbing layer; 0 = off */
  double tau_wall;     /* minimum relaxation time on floor-wall cells (reference default 0.5) */
  double ema_alpha;    /* EMA weight of the time averages, applied at each sample */
  double init_noise;   /* WT_INIT_REST_NOISE: amplitude of the seeded velocity noise */
  int32_t ground;      /* WT_GROUND_* */
  int32_t sides;       /* WT_SIDES_* (3-D z boundaries) */
  int32_t precision;   /* WT_PREC_*; fixed at creation */
  int32_t interp;      /* 1 = Bouzidi interpolated bounce-back (default), 0 = halfway */
  int32_t collision;   /* WT_COLL_* */
  int32_t init_mode;   /* WT_INIT_*: reference free-stream equilibrium, or rest + seeded noise */
  uint32_t init_seed;  /* WT_INIT_REST_NOISE seed */
  uint32_t reserved;
} wt_params;

/* The 96-byte kernel parameter block: Params uniform (src/solver/wgslLbm.ts:6-15) as packed by
 * SolverGPU.writeParams (src/solver/SolverGPU.ts:160-187). */
typedef struct wt_kparams {
  uint32_t nx, ny, nz, n;
  float tau0, csmag2, uin, rho_in;
  uint32_t ground, stride_x;
  float sponge_start, sponge_nu;
  float u_ground, ema_alpha, u_ref;
  uint32_t ref_x;
  uint32_t side_mode, collision;
  float tau_wall;
  uint32_t pad2;
  float sponge_in, contact_h;
  uint32_t interp, stride_p;
} wt_kparams;

/* SolverStats (src/solver/types.ts:31-42), decoded as SolverGPU.stepAndSample does
 * (src/solver/SolverGPU.ts:302-308). raw[] is the 8-slot reduction result:
 * [ΣFx, ΣFy, ΣFz, max|u|², Σρ on x = refX, n_ref, nan count, solid count]. The force sum is
 * accumulated in FP64.
 * Extension (no counterpart in the reference): mass = Σρ over every fluid cell, each cell's density
 * summed in FP64 in a fixed order (the global mass-conservation check), and fluid_cells = the
 * number of cells in that sum. */
typedef struct wt_stats {
  double fx, fy, fz;
  double max_u;
  double rho_ref;
  int64_t step;
  int32_t unstable;
  int32_t reserved;
  double raw[8];
  double mass;
  int64_t fluid_cells;
} wt_stats;

/* WheelDef (src/voxelize/mesh.ts:54-60), grid space. */
typedef struct wt_wheel {
  double c[3];
  double axis[3];
  double r;
  double hw;
} wt_wheel;

/* VoxelInfo (src/voxelize/VoxelizerGPU.ts:6-12). */
typedef struct wt_voxel_info {
  int32_t frontal;
  int32_t solid_cells;
  int32_t min[3];
  int32_t max[3];
} wt_voxel_info;

/* Particle uniform PU (src/render/tracers.ts:5-12) as packed by RendererGPU
 * (src/render/RendererGPU.ts:511-520). */
typedef struct wt_tracer_params {
  uint32_t count, trail, head, emitter; /* emitter: 0 inlet band, 1 rake */
  float steps;
  uint32_t seed;
  float max_age;
  uint32_t nozzles;
  float rake_a[4];
  float rake_b[4];
  uint32_t advance, fill, lines, pad;
  float rake_d[4];
} wt_tracer_params;

/* Streamline uniform SLU (src/render/tracers.ts:152-160) as packed by RendererGPU
 * (src/render/RendererGPU.ts:544-557): seeds = seeds per line x rake lines, points per line,
 * use_mean (0 instantaneous, 1 mean field), per_line = seeds per line; h = step length in cells. */
typedef struct wt_streamline_params {
  uint32_t seeds, points, use_mean, per_line;
  float rake_a[4];
  float rake_b[4];
  float h, p0, p1, p2;
  float rake_d[4];
} wt_streamline_params;

typedef struct wt_solver wt_solver;

/* ---- library ---------------------------------------------------------------------------- */
int wt_version(void);
const char* wt_error_string(int code);
/* Backend.fits (src/backend/webgpu.ts:58-61): bytes the handle would allocate for these dims,
 * and whether they fit in the free memory of the current device (1 yes, 0 no). */
int wt_fits(const wt_dims* dims, int32_t precision, int64_t* bytes_needed, int32_t* fits);
/* SolverGPU.writeParams (src/solver/SolverGPU.ts:160-187). Pure host function. */
int wt_pack_params(const wt_dims* dims, const wt_params* p, wt_kparams* out);

/* ---- solver lifecycle ------------------------------------------------------------------- */
/* SolverFactory (src/backend/types.ts:18) / new SolverGPU (src/solver/SolverGPU.ts:61-144). */
int wt_create(const wt_dims* dims, const wt_params* p, wt_solver** out);
/* LbmSolver.destroy (src/backend/types.ts:15). Accepts NULL. */
void wt_destroy(wt_solver* s);
/* Message of the last failing call on this handle; with s NULL, of the calling thread's last
 * failing call that has no handle (wt_create, wt_fits, wt_sample_noalloc). Valid until the next
 * such call. */
const char* wt_last_error(const wt_solver* s);
/* Backend.setParams (src/backend/types.ts:30) / SolverGPU.setParams (SolverGPU.ts:155-158).
 * precision must equal the creation precision. */
int wt_set_params(wt_solver* s, const wt_params* p);
int wt_get_params(const wt_solver* s, wt_params* out);
int wt_get_kparams(const wt_solver* s, wt_kparams* out);
/* SolverGPU.reset (SolverGPU.ts:190-194): populations re-initialised before the next step. */
int wt_reset(wt_solver* s);
/* SolverGPU.clearStats (SolverGPU.ts:196-201). */
int wt_clear_stats(wt_solver* s);
int64_t wt_step_count(const wt_solver* s);

/* ---- geometry --------------------------------------------------------------------------- */
/* LbmSolver.uploadFlags (types.ts:11): bit 0 solid, bits 8..15 wheel tag k+1. */
int wt_upload_flags(wt_solver* s, const uint32_t* flags, int64_t n);
/* LbmSolver.uploadSdf (types.ts:13) / SolverGPU.uploadSdf (SolverGPU.ts:312-322): wall
 * distances in cells; negative or NaN = unknown. */
int wt_upload_sdf(wt_solver* s, const float* d, int64_t n);
/* SolverGPU.setWheels (SolverGPU.ts:325-335): at most 16 wheels, extra entries are ignored. */
int wt_set_wheels(wt_solver* s, const wt_wheel* w, int32_t count);
/* Backend.voxelize (types.ts:36) / VoxelizerGPU.voxelize (VoxelizerGPU.ts:48-151): voxelizes an
 * indexed triangle mesh (positions xyz f32, u32 indices) through the column-major 4x4 mesh->grid
 * matrix into the solver's flags and wall-distance buffers, tags wheel cells, and returns the
 * frontal projection and bounding box. ntri == 0 clears the geometry. */
int wt_voxelize(wt_solver* s, const float* pos, int64_t nverts, const uint32_t* idx, int64_t ntri,
                const float m[16], const wt_wheel* wheels, int32_t nwheels, wt_voxel_info* info);

/* The same uploads queued the way the reference queues them (SolverGPU.uploadFlags /
 * uploadSdf, SolverGPU.ts:312-322, 342-345: device.queue.writeBuffer, which returns before the
 * copy is done): the copy starts at once on the handle's upload copy stream, overlapping any
 * steps in flight, and the geometry takes effect for every call that follows, exactly as after
 * wt_upload_flags / wt_upload_sdf (unchanged geometry keeps the classification and the captured
 * step graphs). The host buffer must stay valid and unchanged until the next call on the handle
 * that reads or writes the geometry (a step, sample, geometry read, voxelization, tracer,
 * streamline or derived-field call, a synchronous upload, or wt_sync) has returned. The copy
 * overlaps other work only from page-locked host memory. */
int wt_upload_flags_async(wt_solver* s, const uint32_t* flags, int64_t n);
int wt_upload_sdf_async(wt_solver* s, const float* d, int64_t n);

/* ---- time stepping ---------------------------------------------------------------------- */
/* SolverGPU.encodeSteps (SolverGPU.ts:204-222): `steps` fused pull-stream + collide steps. */
int wt_step(wt_solver* s, int32_t steps);
/* SolverGPU.encodePost(enc, false) + result read (SolverGPU.ts:225-247, 292-309): macroscopic
 * fields, EMA statistics, momentum-exchange force and reductions of the current populations. */
int wt_sample(wt_solver* s, wt_stats* out);
/* LbmSolver.stepAndSample (types.ts:14, SolverGPU.ts:292-309). */
int wt_step_and_sample(wt_solver* s, int32_t steps, wt_stats* out);
/* The same call in the reference's asynchronous form (stepAndSample returns a Promise that
 * resolves after sampleBuf.mapAsync, SolverGPU.ts:292-309): wt_step_and_sample_async queues the
 * steps, the sampling pass and the copy of the statistics and returns at once; wt_sample_wait
 * blocks until that sample is done and returns it. Uploads, readbacks and further steps may be
 * queued in between; another sample (wt_sample, wt_step_and_sample, wt_step_and_sample_async,
 * wt_batch_sample) before wt_sample_wait fails with WT_E_STATE, and wt_sample_wait without a
 * pending sample fails with WT_E_STATE. */
int wt_step_and_sample_async(wt_solver* s, int32_t steps);
int wt_sample_wait(wt_solver* s, wt_stats* out);
/* Waits until every queued step, sample, upload and readback of the handle has completed
 * (applying staged asynchronous uploads first). */
int wt_sync(wt_solver* s);

/* ---- readback / checkpoint -------------------------------------------------------------- */
/* SolverGPU.readFlags (SolverGPU.ts:347-356). */
int wt_read_flags(wt_solver* s, uint32_t* out, int64_t n);
/* Encoded wall distances (~bits(d), 0 = unknown) as stored on the device. */
int wt_read_sdf(wt_solver* s, uint32_t* out, int64_t n);
/* SolverGPU.readPopulations (SolverGPU.ts:359-369): the raw current buffer (f32: 4 B, f16: 2 B
 * of f - w, f64: 8 B per population). bytes must equal the buffer size. */
int64_t wt_population_bytes(const wt_solver* s);
int wt_read_populations(wt_solver* s, void* out, int64_t bytes);
/* Checkpoint resume: overwrite the current buffer (same raw layout). Clears any pending reset. */
int wt_write_populations(wt_solver* s, const void* in, int64_t bytes);
/* velTex of the last sample (wgslLbm.ts:439-468): (ux, uy, uz, rho) per cell, stored as FP16 like
 * the reference's rgba16float texture, returned as f32. */
int wt_read_velocity(wt_solver* s, float* out4, int64_t n);
/* The same field in its storage format, the reference texture's rgba16float: 4 IEEE binary16 per
 * cell (8 bytes), copied without widening. */
int wt_read_velocity_half4(wt_solver* s, void* out_half4, int64_t n);
/* The same readback queued (the reference reads its fields through mapAsync, SolverGPU.ts:347-369):
 * the copy starts on the handle's readback copy stream once everything queued so far has
 * completed, and the call returns at once. The next sampling pass that rewrites the field waits
 * for the copy; out_half4 holds the field after wt_sync (or any later call that waits for the
 * handle's work). Overlaps other work only into page-locked host memory. */
int wt_read_velocity_half4_async(wt_solver* s, void* out_half4, int64_t n);
/* meanA (ux, uy, uz, rho EMA, 4 f32 per cell) and meanB (<u.u> EMA, 1 f32 per cell). */
int wt_read_means(wt_solver* s, float* mean4, float* meanb, int64_t n);

/* ---- tracer particles ------------------------------------------------------------------- */
/* PARTICLES_WGSL (src/render/tracers.ts:3-106): one dispatch of the particle kernel against the
 * velocity field of the last sample. Tracer state (count vec4) and trail history (count * trail
 * vec4) live on the device and are (re)allocated when count or trail change (RendererGPU
 * ensureTracers). */
int wt_advect_tracers(wt_solver* s, const wt_tracer_params* p);
int wt_read_tracers(wt_solver* s, float* state4, int64_t count, float* hist4, int64_t hist_len);
int wt_write_tracers(wt_solver* s, const float* state4, int64_t count, const float* hist4,
                     int64_t hist_len, uint32_t trail);

/* ---- derived fields and field export ----------------------------------------------------- */
/* Derived fields (the derived pass, src/solver/wgslLbm.ts:527-592): vorticity (wx, wy, wz) and the
 * Q-criterion (faded out within two cells of a solid) from central differences of the velocity
 * field, turbulence intensity sqrt(k / 3) / uRef from the EMA statistics, and the mean field, as
 * binary16 x 4 per cell (the reference's rgba16float textures), from the velocity field and
 * statistics of the last sample. The first call allocates 24 B per cell. */
int wt_derive_fields(wt_solver* s);
/* Full-resolution read of the derived fields as n x 4 floats; any pointer may be NULL:
 * vort4 = (wx, wy, wz, Q), stat4 = (turbulence intensity, solid, 0, 0), mean4 = the mean field
 * rounded to binary16. Needs a wt_derive_fields call first. */
int wt_read_derived(wt_solver* s, float* vort4, float* stat4, float* mean4, int64_t n);
/* SolverGPU.exportFields (src/solver/SolverGPU.ts:374-425): derives the fields, then reads
 * velocity, mean and vorticity at every stride-th cell (clamped to the last cell) into
 * points = ceil(nx/stride) * ceil(ny/stride) * ceil(nz/stride) float4 each (x fastest); any
 * output pointer may be NULL. */
int wt_export_fields(wt_solver* s, int32_t stride, float* vel4, float* mean4, float* vort4, int64_t points);

/* Streamlines (the streamline pass, src/render/tracers.ts:152-200): seeds x points float4
 * (x, y, z, speed; speed = -1 once the line has ended), seed-major. Mean-field lines use the
 * mean field of the derived pass, which this call runs first. */
int wt_streamlines(wt_solver* s, const wt_streamline_params* p, float* pts4, int64_t n);
/* Probes (the probe pass, src/render/tracers.ts:109-125; Backend.probeData): up to 8 points
 * (pos4: x, y, z, unused) -> out8 per probe: instantaneous (ux, uy, uz, rho) then the mean. Runs
 * the derived pass first for the mean field. */
int wt_probes(wt_solver* s, const float* pos4, int32_t count, float* out8);

/* ---- launch selection (extension; no counterpart in the reference) ------------------------ */
/* Selects the stream-collide launch: `param` cells per thread along x (1, 2 or 4; 2 and 4 need
 * f16/f32 storage and nx % param == 0, otherwise the scalar kernel runs), block bx x by threads
 * (bx * by <= 256; 0, 0 = one row of up to 128 threads), and `kernel` = occupancy hint of the
 * vectorised kernel: 0 = none, 2..4 = registers capped so that many 256-thread CTAs fit on an SM.
 * Until this call or wt_autotune, a handle runs 2 cells per thread, default blocks, and hint 4 for
 * the regularized collision (none for BGK).
 * kernel = WT_LAUNCH_ROW_PIPELINE (param 2, bx 0) selects the row pipeline for D3Q19 with f16 / f32
 * storage: a producer warp streams whole interior rows into shared memory with bulk copies while
 * four consumer warps collide the previous rows; `by` = interior rows per block (0 = 4, at most 16).
 * It needs nx % 8 == 0 (f16) or nx % 4 == 0 (f32) and 3 x 19 x nx populations within 48 KB of
 * shared memory; elsewhere the vectorised kernel runs. */
#define WT_LAUNCH_ROW_PIPELINE 8
/* kernel = WT_LAUNCH_PERSISTENT (param 2, bx 0, by 0): every wt_step call of two or more steps runs
 * as one cooperative launch of a persistent kernel that takes all its steps: per step the resident
 * blocks take the step's work items (wall-cell chunks, face-row tiles, bulk tiles) from an atomic
 * counter, and a grid-wide barrier separates the steps (the same arithmetic as the per-step
 * kernels: bit-identical results). For small grids, where launching a step's kernels costs as much
 * as running them. Needs f16 / f32 storage, nx even and the reference's closure; elsewhere the
 * vectorised kernel runs. */
#define WT_LAUNCH_PERSISTENT 9
/* kernel = WT_LAUNCH_QUEUE (param 2, bx 0, by 0): every step is one launch of that kernel's work
 * queue, one step per launch (no grid barrier, read-only-cache loads), captured in the step graphs
 * like the per-step kernels; the sampling step keeps the per-step kernels. Same conditions and
 * bit-identical results as WT_LAUNCH_PERSISTENT. */
#define WT_LAUNCH_QUEUE 10
int wt_set_launch(wt_solver* s, int32_t kernel, int32_t param, int32_t bx, int32_t by);
int wt_get_launch(const wt_solver* s, int32_t* out4);
/* The project's launch tuner: times every applicable launch candidate on this handle's
 * grid (iters launches each, reading the current populations and writing the other buffer, so
 * the state does not change) and keeps the fastest. out4 (may be NULL) receives
 * {kernel, param, bx, by}. */
int wt_autotune(wt_solver* s, int32_t iters, int32_t* out4);
/* Test hook (extension; no counterpart in the reference): the number of polls each consumer warp of
 * the row pipeline (WT_LAUNCH_ROW_PIPELINE) makes on a stage's barrier before it gives up; polls < 0
 * restores the default (4,194,304). With a small limit the consumers give up while the producer's
 * copies are still in flight: the block stops storing, waits for its copies to land, and sets bit 8
 * of the device error word, which the next sample turns into WT_E_CUDA. Only for tests of that path. */
int wt_set_wait_limit(wt_solver* s, int64_t polls);

/* ---- batches of tunnels ------------------------------------------------------------------- */
/* No counterpart in the reference, whose studies panel runs one tunnel at a time
 * (src/ui/studies.ts:223-252). A batch steps many independent tunnels (any sizes, one device)
 * together: pairs of steps replay one CUDA graph in which every member's step kernels hang off a
 * common fork, so small tunnels run concurrently and one launch advances all of them. Members stay
 * ordinary handles (parameters, geometry and readback work as before; a change of a member's
 * launch, parameters, wheels or geometry makes the batch recapture on its next step). Members must
 * not be used from another thread while a batch call runs, and must outlive the batch. */
typedef struct wt_batch wt_batch;
int wt_batch_create(wt_solver* const* members, int32_t count, wt_batch** out);
void wt_batch_destroy(wt_batch* b); /* the members stay alive */
const char* wt_batch_last_error(const wt_batch* b);
int32_t wt_batch_size(const wt_batch* b);
/* `steps` lattice updates of every member */
int wt_batch_step(wt_batch* b, int32_t steps);
/* the sampling pass of every member (queued together, then read back): out has count entries */
int wt_batch_sample(wt_batch* b, wt_stats* out);
/* on = 1: when every member is D3Q19 with the same f16 / f32 storage and collision, no learned
 * closure and the vectorised launch, the bulk rows of all members step in one launch of a batch
 * kernel over a table of per-tunnel descriptors (face rows and wall cells stay per member).
 * on = WT_BATCH_PERSISTENT: when every member has the same lattice, f16 / f32 storage and collision,
 * no learned closure and an even nx (at most 48 members), each wt_batch_step call of two or more
 * steps is one cooperative launch of the persistent kernel over all members: per step the resident
 * blocks take the wall-cell chunks, face-row tiles and bulk tiles of every member from an atomic
 * counter, with a grid-wide barrier between steps. Members stay bit-identical to the same handles
 * stepped alone.
 * on = WT_BATCH_QUEUE: under the same conditions, every step of every member is one launch of the
 * same work queue (resident blocks taking wall chunks, face tiles and bulk tiles of all members
 * from an atomic counter), without the grid barrier: the steps are separate launches, captured in
 * the batch's CUDA graphs, so the population loads keep the read-only cache path. Members stay
 * bit-identical to the same handles stepped alone.
 * on = 0 (default): the members' own kernels under one graph. */
#define WT_BATCH_PERSISTENT 2
#define WT_BATCH_QUEUE 3
int wt_batch_set_fused(wt_batch* b, int32_t on);

/* ---- learned LES closure (extension; no counterpart in the reference) -----------------------
 * A per-cell network replaces the Smagorinsky eddy viscosity of the collision (the reference's
 * closure: wgslLbm.ts:206-214) on D3Q19 handles with f16 or f32 storage. Its 10 features per
 * cell, in the handle's lattice units, from the pre-collision populations:
 *   0-5  non-equilibrium stress Pi_xx, Pi_yy, Pi_zz, Pi_xy, Pi_xz, Pi_yz
 *        (Pi = sum_i c_i c_i f_i - rho (u u + I / 3))
 *   6    |S| = 3 |Pi| / (sqrt(2) rho tau_s), tau_s = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi| / rho)) / 2
 *        with Cs = WT_CLOSURE_FEATURE_CS and |Pi| = sqrt(Pi : Pi): the strain rate the Smagorinsky
 *        relation assigns to the stress
 *   7    wall distance in cells from the handle's wall-distance field, WT_CLOSURE_WALL_CAP where
 *        unknown or larger
 *   8    rho
 *   9    |u|
 * Network 10 -> 32 -> 32 -> 1: x' = bf16((x - shift) * scale); h1 = bf16(gelu(x' W1 + b1));
 * h2 = bf16(gelu(h1 W2 + b2)); nu_t = nu_scale * softplus(h2 . w3 + b3), with W1, W2, w3 rounded
 * to bf16, f32 accumulation and gelu(x) = x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))) / 2.
 * The relaxation time becomes tau = tau0' + 3 nu_t, tau0' being tau0 with the outlet sponge and
 * the floor-wall minimum exactly as for Smagorinsky. */
#define WT_CLOSURE_IN 10
#define WT_CLOSURE_HID 32
#define WT_CLOSURE_FEATURE_CS 0.1f
#define WT_CLOSURE_WALL_CAP 3.0f
typedef struct wt_closure {
  float shift[WT_CLOSURE_IN]; /* feature normalisation x' = (x - shift) * scale */
  float scale[WT_CLOSURE_IN];
  float w1[WT_CLOSURE_IN][WT_CLOSURE_HID]; /* [input][hidden] */
  float b1[WT_CLOSURE_HID];
  float w2[WT_CLOSURE_HID][WT_CLOSURE_HID]; /* [hidden in][hidden out] */
  float b2[WT_CLOSURE_HID];
  float w3[WT_CLOSURE_HID];
  float b3;
  float nu_scale; /* output scale (lattice viscosity units) */
} wt_closure;
/* Installs the network (copied) on the handle, or removes it (closure = NULL: plain Smagorinsky).
 * WT_E_UNSUPPORTED on D2Q9 and f64 handles. */
int wt_set_closure(wt_solver* s, const wt_closure* closure);
/* enabled = 1 and *out = the installed network, or enabled = 0 */
int wt_get_closure(const wt_solver* s, wt_closure* out, int32_t* enabled);

/* Trainer of the closure: a device-resident pool of samples (features + target eddy viscosity),
 * the network's f32 master weights and Adam state, and the BF16 training kernels (tcgen05 forward,
 * input-gradient and weight-gradient products, f32 accumulation). One trainer per device; calls on one trainer are
 * serialized by the caller. */
typedef struct wt_trainer wt_trainer;
typedef struct wt_train_params {
  int32_t steps;  /* Adam steps */
  int32_t batch;  /* samples per step, drawn uniformly with replacement from the pool */
  float lr, beta1, beta2, eps;
  uint64_t seed;  /* minibatch draws */
} wt_train_params;
int wt_trainer_create(int32_t device, int64_t capacity, wt_trainer** out);
void wt_trainer_destroy(wt_trainer* t);
const char* wt_trainer_last_error(const wt_trainer* t);
int64_t wt_trainer_count(const wt_trainer* t);
int wt_trainer_clear(wt_trainer* t);
/* Appends training samples from a fine run and the coarse grid it is filtered to (fine dims = 2 x
 * coarse dims; both D3Q19, same body voxelized on each). Each coarse fluid cell whose 2 x 2 x 2
 * fine cells are all fluid, outside both sponges and off the domain faces, is kept with
 * probability `keep` (a hash of the cell and `seed`). Its features are those of the box-filtered
 * fine populations (pulled, pre-collision) seen by the coarse handle (its tau0 and wall distances);
 * its target is the eddy viscosity that best represents the unresolved stress:
 *   T = <rho u u> / <rho> - u~ u~  +  <-2 nu_sgs S>   (filtered resolved stress plus the fine run's
 *       own Smagorinsky stress; < > = 2 x 2 x 2 average, u~ = <rho u> / <rho>)
 *   nu* = max(0, -sum_box dev(T) : S~ / sum_box 2 S~ : S~), S~ from central differences of u~ on the
 *       coarse grid, sums over the 3 x 3 x 3 coarse neighbourhood (see
 *       wt_trainer_set_projection_radius) of cells with a full stencil. added (may be NULL) receives the number of samples appended. */
int wt_trainer_add_samples(wt_trainer* t, wt_solver* fine, wt_solver* coarse, double keep, uint64_t seed,
                           int64_t* added);
/* half-width of the projection box of later wt_trainer_add_samples calls: the sums run over
 * (2 radius + 1)^3 coarse cells (1, the default, to 3); kept cells lie radius + 1 cells off the
 * faces */
int wt_trainer_set_projection_radius(wt_trainer* t, int32_t radius);
/* host samples: x (n x 10 features), y (n targets) */
int wt_trainer_put_samples(wt_trainer* t, const float* x, const float* y, int64_t n);
int wt_trainer_read_samples(wt_trainer* t, int64_t offset, int64_t n, float* x, float* y);
/* mean and standard deviation of the 10 features and the target over the pool (11 each) */
int wt_trainer_stats(wt_trainer* t, double* mean11, double* std11);
int wt_trainer_set_model(wt_trainer* t, const wt_closure* m); /* also resets the Adam state */
int wt_trainer_get_model(const wt_trainer* t, wt_closure* out);
/* Adam on L = mean(((nu_t(x) - y) / nu_scale)^2); loss (may be NULL) receives the minibatch loss of
 * every step. */
int wt_trainer_fit(wt_trainer* t, const wt_train_params* p, float* loss);
/* loss and gradient (dL / d parameter, in a wt_closure whose shift, scale and nu_scale are 0) over
 * pool samples [offset, offset + n), without an update */
int wt_trainer_grad(wt_trainer* t, int64_t offset, int64_t n, wt_closure* grad, double* loss);
/* nu_t of the current model for n host feature rows (the tensor-core inference path) */
int wt_trainer_infer(wt_trainer* t, const float* x, int64_t n, float* nu);

/* ---- device plumbing -------------------------------------------------------------------- */
/* The handle's cudaStream_t (for event timing by the caller) and its device ordinal. */
void* wt_stream(const wt_solver* s);
int32_t wt_device(const wt_solver* s);
/* Number of kernel launches this handle has issued since creation. */
int64_t wt_launch_count(const wt_solver* s);
/* Number of wt_step_and_sample calls whose last step ran the sampling pass fused (extension). With
 * f16 / f32 storage, the vectorised kernels and the reference's closure, the last step of a
 * stepAndSample chunk writes the velocity texels, the EMA statistics and the sums of the sampling
 * pass from the values it stores, and a short pass over the wall-adjacent and solid cells adds the
 * momentum-exchange force: the populations are not read a second time. The statistics, the
 * velocity field and the means are bit-identical to wt_step followed by wt_sample (the force sums
 * to FP64 rounding, summed in another order). Other configurations run the separate pass. */
int64_t wt_fused_sample_count(const wt_solver* s);

/* ---- sampling pass on caller-owned buffers, without allocating ------------------------------
 * No counterpart in the reference: the reference's solver always owns its buffers.
 *
 * For callers that may not allocate device memory: hosts whose device memory all belongs to
 * another allocator (a framework's caching allocator, or an arena reserved at start-up). Such a
 * host must not call cudaMalloc / cudaFree, because those calls synchronise the whole device and
 * take memory that the owning allocator does not account for. It keeps the tunnel's buffers in
 * its own memory and runs the sampling pass on them here: velocity field, EMA statistics,
 * momentum-exchange force and the reductions, as wt_sample does for a handle. The call allocates
 * nothing: no cudaMalloc, no cudaFree, no allocating library routine.
 *
 * The pass needs a reduction scratch of one 80-byte slot per 256 cells. It is a fixed array in
 * the library's device memory (1.25 MiB per device), so grids are limited to
 * WT_SAMPLE_NOALLOC_MAX_CELLS cells; larger grids are rejected with WT_E_INVALID.
 *
 * Buffers: device memory of the device current on the calling thread, laid out as a handle's:
 *   populations  q * n values in the storage format of p->precision (f16 holds f - w)
 *   flags        n u32 (bit 0 solid, bits 8-15 wheel tag)
 *   sdf_encoded  n u32, ~bits(distance) and 0 where unknown (the format of wt_read_sdf)
 *   vel_half4    n x 4 binary16 (ux, uy, uz, rho), written
 *   mean4, meanb n x 4 and n floats of EMA state, read and rewritten (a handle starts them at
 *                (0, 0, 0, 1) and 0)
 *   result8      8 doubles, written: the raw reduction of wt_stats.raw
 * wheels (host array, up to 16) and p are read during the call only. The kernels are queued on
 * `stream` (NULL: the default stream) and the call returns without waiting for them.
 *
 * The first call on a device looks up the scratch array's address (cudaGetSymbolAddress), which
 * can load the library's device code; make that first call before any stream capture. Every call
 * shares the one array and it keeps the last call's contents; a call writes every slot it reads
 * before reading it, so nothing has to be cleared. Calls that overlap on the GPU (streams with no
 * ordering between them) race on the array: order them on one stream or with events.
 * Errors: WT_E_INVALID, WT_E_NO_DEVICE, WT_E_CUDA; the message is in wt_last_error(NULL). */
#define WT_SAMPLE_NOALLOC_MAX_CELLS 4194304
int wt_sample_noalloc(const wt_dims* dims, const wt_params* p, const wt_wheel* wheels, int32_t nwheels,
                      const void* populations, const uint32_t* flags, const uint32_t* sdf_encoded, void* vel_half4,
                      float* mean4, float* meanb, double* result8, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WT_H */
