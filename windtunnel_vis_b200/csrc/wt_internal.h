// wt_internal.h — handle layout and kernel launchers shared by the translation units of libwt.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/wt.h"
#include "wt_closure.cuh"
#include "wt_common.cuh"

// step pairs captured in one long step graph
constexpr int WT_LONG_PAIRS = 5;
// steps in the captured tail of a stepAndSample chunk (even: the graph keeps the parity)
constexpr int WT_SAMPLE_TAIL = 10;
// doubles per block in the macro pass's partial reductions, and in its result: the reference's
// 8-slot result followed by the FP64 fluid mass and the fluid cell count
constexpr int MACRO_SLOTS = 10;
constexpr size_t RESULT_BYTES = MACRO_SLOTS * sizeof(double);

struct wt_solver {
  int device = 0;
  int num_sms = 148;  // streaming multiprocessors of `device` (persistent grids)
  cudaStream_t stream = nullptr;
  // the face-row and per-cell boundary kernels run on `aux`, forked from and joined back into
  // `stream` around each step, so they overlap the bulk kernel
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // two-step (one ping-pong cycle) CUDA graphs, one per starting parity; rebuilt after any change
  // of launch shape, parameters, wheels or boundary list
  cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
  int64_t graph_launches = 0;  // kernel launches inside one graph replay
  // the same for 2 x WT_LONG_PAIRS steps: fewer graph launches per reference sample chunk
  cudaGraphExec_t long_graph[2] = {nullptr, nullptr};
  int64_t long_graph_launches = 0;
  // the tail of a stepAndSample chunk: WT_SAMPLE_TAIL - 1 steps, then the fused sampling step (with
  // its wall-force pass and final reduction), per starting parity
  cudaGraphExec_t sample_graph[2] = {nullptr, nullptr};
  int64_t sample_graph_launches = 0;
  uint64_t graph_gen = 0;      // bumped whenever the captured graphs are dropped (batches recapture)
  wt_dims dims{};
  wt_params params{};
  wt_kparams kp{};
  int prec = WT_PREC_F32;
  int q = 9;
  bool is3d = false;
  size_t n = 0;
  size_t pop_elem = 4;  // bytes per stored population
  void* f[2] = {nullptr, nullptr};
  int parity = 0;  // current populations in f[parity]
  int64_t step_count = 0;
  bool pending_init = true;
  uint32_t* flags = nullptr;
  uint32_t* sdf = nullptr;
  // uploads land here first and replace flags / sdf only when their content differs, so that
  // re-uploading unchanged geometry keeps the classification and the captured graphs
  uint32_t* stage = nullptr;
  uint32_t* diff_dev = nullptr;   // device words: a staged buffer differs from the current one
  uint32_t* diff_host = nullptr;  // pinned copies (written by k_take_word through their mapping)
  uint32_t* diff_host_dev = nullptr;  // device address of diff_host
  uint8_t* cls = nullptr;
  bool cls_dirty = true;
  bool tab_dirty = false;  // link records need a rebuild (parameters or wheels changed)
  // cells the vectorised bulk kernel leaves to the boundary kernel: every cell of an aligned group
  // of `gs` cells along x that holds a solid cell, a fluid cell next to a solid, or lies on a
  // domain face (built by launch_classify)
  uint32_t* bnd = nullptr;
  uint32_t nbnd = 0;
  size_t bnd_cap = 0;
  int gs = 1;
  // every solid cell (built with the boundary list): the fused sampling pass visits them after the
  // sampling step (density extrapolation, velocity texel, EMA statistics)
  uint32_t* solids = nullptr;
  uint32_t nsolid = 0;
  size_t solid_cap = 0;
  // accumulator sets of the fused sampling pass (zeroed before each sampling step)
  unsigned long long* smp_sets = nullptr;
  int64_t fused_samples = 0;  // stepAndSample calls that ran the fused sampling step
  unsigned* ps_bar = nullptr;  // grid barrier words of the persistent kernel (WT_LAUNCH_PERSISTENT)
  uint32_t* bnd_count = nullptr;  // device counter used while building the list
  uint32_t* bnd_count_host = nullptr;  // pinned
  // link records of the listed cells (k_boundary_build), applied every step by k_boundary_tab
  uint2* bcell = nullptr;  // {cell, BC_* bits} per listed cell
  uint4* brec = nullptr;   // {a1, a2, alpha, beta} per link
  float* bgam = nullptr;   // gamma per link
  size_t btab_cap = 0;     // cells the record buffers hold
  // solid cells of f[b] hold the rest state (the reference rewrites them every step; here they
  // are written once per buffer after a classification or a raw population write)
  bool solid_ok[2] = {false, false};
  uint2* vel = nullptr;  // half4 (ux, uy, uz, rho) per cell
  float4* vel_f32 = nullptr;  // f32 copy of `vel` for readback, allocated by the first wt_read_velocity
  float4* meanA = nullptr;
  float* meanB = nullptr;
  double* partials = nullptr;  // per-block partial reductions of the macro pass
  int partial_blocks = 0;
  double* result_dev = nullptr;  // MACRO_SLOTS doubles
  double* result_host = nullptr; // pinned
  wt::Wheels wheels{};
  // derived fields (binary16 x 4 per cell, allocated by the first wt_derive_fields): vorticity and
  // Q, turbulence intensity and the solid mask, the mean field; and the export staging buffer
  uint2* dvort = nullptr;
  uint2* dstat = nullptr;
  uint2* dmean = nullptr;
  float4* exp_buf = nullptr;
  size_t exp_cap = 0;  // float4 elements
  float4* probe_buf = nullptr;  // 8 positions + 16 results
  // voxelizer: device copies of the last mesh (grown as needed) and the 8-word info block
  void* vox_pos = nullptr;
  void* vox_idx = nullptr;
  size_t vox_pos_cap = 0, vox_idx_cap = 0;
  uint32_t* vox_info = nullptr;
  // tracers
  float4* tr_state = nullptr;
  float4* tr_hist = nullptr;
  uint32_t tr_count = 0, tr_trail = 0;
  // stream-collide launch (chosen per lattice by the tuner, see wt_lbm.cu): sc_param cells per
  // thread along x (1 = scalar kernel), block sc_bx x sc_by of the vectorised kernel (0 = default)
  int block_x = 0;
  int sc_kernel = 0, sc_param = 2, sc_bx = 0, sc_by = 0;
  // polls of each row-pipeline consumer wait before it gives up (wt_set_wait_limit)
  uint32_t rp_wait_limit = 1u << 22;
  // false until wt_set_launch or wt_autotune chose a launch: the default then follows the collision
  // operator (occupancy hint 4 for the regularized collision, which fits 64 registers; none for BGK)
  bool launch_explicit = false;
  // learned closure (wt_set_closure): device copy of the network, nullptr = Smagorinsky
  wt::ClosureDev* closure_dev = nullptr;
  wt::ClosureParams closure_p{};  // the network's small values, passed by value to the kernels
  wt_closure closure_host{};
  // the learned closure's face rows and wall cells: their features ([rows][10]) followed by their
  // eddy viscosities ([rows]), rows = face cells + boundary-table capacity
  float* lc_rows = nullptr;
  size_t lc_rows_cap = 0;
  int* err_dev = nullptr;   // device-side error word written by kernels with bounded waits
  int* err_host = nullptr;  // pinned copy
  int64_t launches = 0;
  // asynchronous transfers (wt_*_async, created by the first such call): one copy stream per
  // direction, so that an upload and a readback overlap each other and the compute stream
  cudaStream_t copy_up = nullptr, copy_rd = nullptr;
  uint32_t* stage_flags = nullptr;  // staged asynchronous uploads, applied by settle_uploads
  uint32_t* stage_sdf = nullptr;
  bool up_flags = false, up_sdf = false;  // a staged upload waits to be applied
  cudaEvent_t ev_up = nullptr;   // on copy_up: after the last asynchronous upload and its comparison
  cudaEvent_t ev_swap = nullptr; // on stream: after the steps that may read a buffer swapped out
  bool swap_pending = false;     // the next asynchronous upload waits for ev_swap
  cudaEvent_t ev_src = nullptr;  // on stream: the state an asynchronous readback copies
  cudaEvent_t ev_rd = nullptr;   // on copy_rd: after the last asynchronous readback
  bool rd_issued = false;        // ev_rd has been recorded: writers of `vel` wait for it
  cudaEvent_t ev_smp = nullptr;  // on stream: after the result copy of an asynchronous sample
  bool sample_pending = false;   // wt_step_and_sample_async issued, wt_sample_wait not yet called
  int64_t sample_step = 0;       // step count of the last queued sample (its statistics' `step`)
  std::string err;
};

namespace wt {

int lbm_block_x(const wt_solver* s);
// sizes the learned closure's row buffer for the current lattice and boundary table (outside
// graph capture); true in *grown when it was reallocated
cudaError_t closure_rows_reserve(wt_solver* s, bool* grown);
// dynamic shared memory of the row-pipeline bulk kernel on this handle, 0 where it does not apply
size_t rows_pipeline_smem(const wt_solver* s);
cudaError_t launch_classify(wt_solver* s);
cudaError_t launch_boundary_table(wt_solver* s);
cudaError_t launch_init(wt_solver* s);
cudaError_t launch_stream_collide(wt_solver* s, const void* fin, void* fout);
cudaError_t launch_macro(wt_solver* s);
// The fused sampling step (the last step of a stepAndSample chunk runs the sampling pass's per-cell
// work on what it stores, then the wall-force / solid-cell pass and the final reduction into
// result_dev). sample_step_ok: whether the handle's step takes that form (vectorised kernels, f16 /
// f32 storage, the reference's closure, not the row pipeline); needs a classified handle.
bool sample_step_ok(const wt_solver* s);
cudaError_t launch_sample_step(wt_solver* s, const void* fin, void* fout);
constexpr size_t SMP_SETS_BYTES = 64 * 16 * sizeof(unsigned long long);

// voxelizer (wt_voxel.cu). Scratch buffers hits (3n i32), vote (n u32), info (8 u32) are
// allocated by the caller.
struct VoxelJob {
  const float* pos;     // device, 3 * nverts
  const uint32_t* idx;  // device, 3 * ntri
  int64_t ntri;
  float M[16];
  int32_t* hits;
  uint32_t* vote;
  uint32_t* info;
};
cudaError_t launch_voxelize(wt_solver* s, const VoxelJob& job);

// Batches (wt_lbm.cu): the bulk rows of every tunnel of a batch in one launch. A tunnel's blocks
// are tiles of BATCH_BX x BATCH_BY threads (two cells per thread along x); tile0 is the prefix of
// the tile counts. The table travels by value (constant bank).
constexpr int BATCH_MAX_FUSED = 64;
constexpr int BATCH_BX = 64, BATCH_BY = 2;
struct BatchTunnel {
  wt_kparams P;
  const void* fin;
  void* fout;
  const uint8_t* cls;
  int gs;
  uint32_t tiles_x, tiles_y, pad;
};
struct BatchTable {
  uint32_t count;
  uint32_t tile0[BATCH_MAX_FUSED + 1];
  BatchTunnel t[BATCH_MAX_FUSED];
};
// whether a handle's step can join the batch kernel: D3Q19, f16 / f32, vectorised path, no closure
bool batch_fusable(const wt_solver* s);
// The persistent kernel: `steps` updates of the tunnels ms[0 .. count) (same lattice, storage and
// collision; each persistent_ok) in one cooperative launch on `st`; bar = PS_BAR_WORDS device words
// (zeroed here: the grid barrier's two and the work counters of two consecutive steps), err = the
// device error word for a barrier timeout (bit 16). The members' parities are not changed here.
constexpr int PS_BAR_WORDS = 4;
bool persistent_ok(const wt_solver* s);
cudaError_t launch_persistent(wt_solver* const* ms, int count, int steps, unsigned* bar, int* err, cudaStream_t st);
// one step of every tunnel in one launch of the persistent kernel's work queue (read-only-cache
// loads, no grid barrier), step k0 of a graph: the tunnels start at parity parity ^ (k0 & 1), and the
// launch takes item counter bar[2 + (k0 & 1)] and clears the other
cudaError_t launch_queue_step(wt_solver* const* ms, int count, int k0, unsigned* bar, int* err, cudaStream_t st);
// the face-row and wall-cell kernels of one step of `s` on its auxiliary stream, forked from
// `origin`; s->ev_join is recorded at their end (the caller joins it into `origin`)
cudaError_t launch_aux_kernels(wt_solver* s, const void* fin, void* fout, cudaStream_t origin);
// the batch kernel over `tab` (all members: precision `prec`, collision `bgk`)
cudaError_t launch_batch_bulk(int prec, bool bgk, const BatchTable& tab, uint32_t tiles, cudaStream_t st);

// learned closure training data (wt_lbm.cu): the fine handle's current populations box-filtered
// onto a cnx x cny x cnz grid (fine dims = 2 x coarse dims); `out` holds 11 * cnx * cny * cnz floats
cudaError_t launch_closure_filter(wt_solver* fine, int cnx, int cny, int cnz, float* out, cudaStream_t st);

// derived fields and export (wt_fields.cu)
cudaError_t launch_derive(wt_solver* s);
cudaError_t launch_export(wt_solver* s, int stride, int ox, int oy, int oz, float4* out);
cudaError_t launch_widen_half4(wt_solver* s, const uint2* src, float4* dst, size_t n);

// tracers, streamlines and probes (wt_tracer.cu)
cudaError_t launch_tracers(wt_solver* s, const wt_tracer_params& p);
cudaError_t launch_streamlines(wt_solver* s, const wt_streamline_params& p, float4* pts);
cudaError_t launch_probes(wt_solver* s, const float4* pos, int count, float4* out);

// records `msg` as the calling thread's message for wt_last_error(NULL) and returns `code`
int fail_unbound(int code, const std::string& msg);

}  // namespace wt
