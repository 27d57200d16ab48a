// wt_api.cu — the extern "C" entry points of libwt.so (declared in include/wt.h).
//
// One handle = one tunnel on the device that was current at creation, with its own stream. The
// handle owns every device buffer; host pointers passed in are only read/written during the
// call. Errors never abort: each entry point returns a WT_E_* code and records a message.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "wt_internal.h"
#include "wt_closure.cuh"

namespace {

thread_local std::string g_create_err;

int fail(wt_solver* s, int code, const std::string& msg) {
  if (s) s->err = msg;
  else g_create_err = msg;
  return code;
}

int cuda_fail(wt_solver* s, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a non-sticky error
  return fail(s, e == cudaErrorMemoryAllocation ? WT_E_OOM : WT_E_CUDA, m);
}

#define WT_CUDA(s, call, what)                         \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(s, e_, what); \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

size_t elem_bytes(int prec) { return prec == WT_PREC_F16 ? 2 : (prec == WT_PREC_F64 ? 8 : 4); }

bool dims_ok(const wt_dims* d) {
  if (!d || d->nx < 1 || d->ny < 1 || d->nz < 1) return false;
  if (d->ny > 65535 || d->nz > 65535) return false;  // grid.y / grid.z of the row launches
  const uint64_t n = (uint64_t)d->nx * (uint64_t)d->ny * (uint64_t)d->nz;
  return n < (1ull << 32);  // the kernel parameter block carries n as u32, like the reference
}

int64_t bytes_for(const wt_dims* d, int prec) {
  const int64_t n = (int64_t)d->nx * d->ny * d->nz;
  const int64_t q = d->nz > 1 ? 19 : 9;
  // 2 population buffers + flags + sdf + upload stage + class byte + half4 velocity + meanA + meanB
  return n * (2 * q * (int64_t)elem_bytes(prec) + 4 + 4 + 4 + 1 + 8 + 16 + 4);
}

void free_all(wt_solver* s) {
  void* bufs[] = {s->f[0], s->f[1], s->flags, s->sdf, s->cls, s->vel, s->vel_f32, s->meanA, s->meanB,
                  s->partials, s->result_dev, s->err_dev, s->tr_state, s->tr_hist, s->bnd, s->bnd_count,
                  s->bcell, s->brec, s->bgam, s->vox_pos, s->vox_idx, s->vox_info,
                  s->dvort, s->dstat, s->dmean, s->exp_buf, s->probe_buf, s->closure_dev, s->stage,
                  s->diff_dev, s->lc_rows, s->solids, s->smp_sets, s->ps_bar, s->stage_flags, s->stage_sdf};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (s->result_host) cudaFreeHost(s->result_host);
  if (s->err_host) cudaFreeHost(s->err_host);
  if (s->bnd_count_host) cudaFreeHost(s->bnd_count_host);
  if (s->diff_host) cudaFreeHost(s->diff_host);
  for (auto& g : s->step_graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : s->long_graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : s->sample_graph)
    if (g) cudaGraphExecDestroy(g);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  for (cudaEvent_t e : {s->ev_up, s->ev_src, s->ev_rd, s->ev_smp, s->ev_swap})
    if (e) cudaEventDestroy(e);
  if (s->copy_up) cudaStreamDestroy(s->copy_up);
  if (s->copy_rd) cudaStreamDestroy(s->copy_rd);
  if (s->aux) cudaStreamDestroy(s->aux);
  if (s->stream) cudaStreamDestroy(s->stream);
}

// The auxiliary stream gets the highest priority so that the block scheduler dispatches the
// small, latency-bound face / boundary kernels ahead of the bulk kernel's queued blocks.
cudaError_t create_priority_stream(cudaStream_t* st) {
  int lo = 0, hi = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (e != cudaSuccess) return e;
  return cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, hi);
}

// Drops the captured step graphs (they bake in the launch shape, the parameter block, the wheels
// and the boundary list); the next wt_step recaptures them.
void invalidate_graphs(wt_solver* s) {
  for (auto& g : s->step_graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  for (auto& g : s->long_graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  for (auto& g : s->sample_graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  s->graph_gen++;
}

// ---- small device helpers used only by the API -----------------------------------------------
__global__ void k_encode_sdf(uint32_t* __restrict__ buf, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = __uint_as_float(buf[i]);
    buf[i] = v >= 0.0f ? ~__float_as_uint(v) : 0u;  // negative or NaN -> unknown
  }
}

// *out |= 1 if a and b differ anywhere
__global__ void k_diff_words(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, size_t n,
                             uint32_t* __restrict__ out) {
  bool d = false;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d = d || a[i] != b[i];
  if (__syncthreads_or(d) && threadIdx.x == 0) atomicOr(out, 1u);
}

// *host = *word, then *word = 0: the difference word reaches the host through mapped page-locked
// memory (a store over the bus, not a copy-engine transfer, so it never queues behind a large
// asynchronous readback), and the word is clear for the next comparison
__global__ void k_take_word(uint32_t* __restrict__ word, volatile uint32_t* host) {
  *host = *word;
  *word = 0u;
}

__global__ void k_clear_stats(float4* __restrict__ meanA, float* __restrict__ meanB, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    meanA[i] = make_float4(0.f, 0.f, 0.f, 1.f);
    meanB[i] = 0.f;
  }
}

__global__ void k_vel_to_f32(const uint2* __restrict__ vel, float4* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint2 v = vel[i];
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    out[i] = make_float4(a.x, a.y, b.x, b.y);
  }
}

unsigned grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

// Class bytes, boundary list and link records after a geometry change; link records alone after a
// change of parameters or wheels (they hold the wall and inlet terms).
int ensure_classified(wt_solver* s) {
  if (s->cls_dirty) {
    invalidate_graphs(s);
    WT_CUDA(s, wt::launch_classify(s), "classify");
    s->cls_dirty = false;
    s->tab_dirty = false;
  } else if (s->tab_dirty) {
    invalidate_graphs(s);
    WT_CUDA(s, wt::launch_boundary_table(s), "boundary links");
    s->tab_dirty = false;
  }
  if (s->closure_dev) {
    bool grown = false;
    WT_CUDA(s, wt::closure_rows_reserve(s, &grown), "closure rows");
    if (grown) invalidate_graphs(s);
  }
  return WT_OK;
}

// Captures `pairs` ping-pong step pairs for starting parity p (f[p] -> f[p^1] -> f[p], repeated)
// into *out; *launches receives the kernel launches of one replay.
int capture_steps(wt_solver* s, int p, int pairs, cudaGraphExec_t* out, int64_t* launches) {
  const int64_t l0 = s->launches;
  cudaGraph_t graph = nullptr;
  WT_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < pairs && e == cudaSuccess; k++) {
    e = wt::launch_stream_collide(s, s->f[p], s->f[p ^ 1]);
    if (e == cudaSuccess) e = wt::launch_stream_collide(s, s->f[p ^ 1], s->f[p]);
  }
  cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
  *launches = s->launches - l0;
  s->launches = l0;
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, graph, cudaGraphInstantiateFlagUseNodePriority);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(s, e, "graph capture");
  }
  return WT_OK;
}

// the two-step graph for starting parity p: step f[p] -> f[p^1], then f[p^1] -> f[p]
int capture_step_graph(wt_solver* s, int p) { return capture_steps(s, p, 1, &s->step_graph[p], &s->graph_launches); }

// the tail of a stepAndSample chunk for starting parity p: WT_SAMPLE_TAIL - 1 steps, then the fused
// sampling step (ending on f[p]: the tail has an even number of steps)
int capture_sample_graph(wt_solver* s, int p) {
  const int64_t l0 = s->launches;
  cudaGraph_t graph = nullptr;
  WT_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
  cudaError_t e = cudaSuccess;
  int q = p;
  for (int k = 0; k < WT_SAMPLE_TAIL - 1 && e == cudaSuccess; k++, q ^= 1)
    e = wt::launch_stream_collide(s, s->f[q], s->f[q ^ 1]);
  if (e == cudaSuccess) e = wt::launch_sample_step(s, s->f[q], s->f[q ^ 1]);
  cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
  s->sample_graph_launches = s->launches - l0;
  s->launches = l0;
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s->sample_graph[p], graph, cudaGraphInstantiateFlagUseNodePriority);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    s->sample_graph[p] = nullptr;
    return cuda_fail(s, e, "graph capture");
  }
  return WT_OK;
}

int ensure_init(wt_solver* s) {
  if (!s->pending_init) return WT_OK;
  WT_CUDA(s, wt::launch_init(s), "init");
  s->pending_init = false;
  s->solid_ok[0] = s->solid_ok[1] = true;  // init writes the rest state into solid cells
  return WT_OK;
}

// Reads (and clears) the device error word set by kernels whose bounded waits gave up.
int check_err_flag(wt_solver* s) {
  WT_CUDA(s, cudaMemcpyAsync(s->err_host, s->err_dev, 4, cudaMemcpyDeviceToHost, s->stream), "read error word");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read error word");
  if (*s->err_host != 0) {
    const int code = *s->err_host;
    *s->err_host = 0;
    cudaMemsetAsync(s->err_dev, 0, 4, s->stream);
    return fail(s, WT_E_CUDA, "a kernel's bounded wait timed out (device error word " + std::to_string(code) + ")");
  }
  return WT_OK;
}

void decode(const wt_solver* s, const double* d, wt_stats* out) {
  std::memset(out, 0, sizeof *out);
  for (int k = 0; k < 8; k++) out->raw[k] = d[k];
  out->mass = d[8];
  out->fluid_cells = (int64_t)d[9];
  out->fx = d[0];
  out->fy = d[1];
  out->fz = d[2];
  out->max_u = std::sqrt(d[3] > 0 ? d[3] : 0.0);
  out->rho_ref = d[5] > 0 ? d[4] / d[5] : 1.0;
  out->unstable = (d[6] > 0 || !std::isfinite(d[0]) || d[3] > 0.25) ? 1 : 0;
  out->step = s->sample_step;
}

}  // namespace

namespace wt {
int fail_unbound(int code, const std::string& msg) { return fail(nullptr, code, msg); }
}  // namespace wt

extern "C" {

int wt_version(void) { return WT_ABI_VERSION; }

const char* wt_error_string(int code) {
  switch (code) {
    case WT_OK: return "ok";
    case WT_E_INVALID: return "invalid argument";
    case WT_E_CUDA: return "CUDA error";
    case WT_E_OOM: return "out of device memory";
    case WT_E_STATE: return "invalid state";
    case WT_E_UNSUPPORTED: return "unsupported";
    case WT_E_NO_DEVICE: return "no CUDA device";
    default: return "unknown error";
  }
}

int wt_pack_params(const wt_dims* d, const wt_params* p, wt_kparams* k) {
  if (!d || !p || !k) return WT_E_INVALID;
  std::memset(k, 0, sizeof *k);
  const uint32_t nx = (uint32_t)d->nx, ny = (uint32_t)d->ny, nz = (uint32_t)d->nz;
  k->nx = nx;
  k->ny = ny;
  k->nz = nz;
  k->n = nx * ny * nz;
  k->tau0 = (float)(3.0 * p->nu + 0.5);
  k->csmag2 = (float)(p->cs * p->cs);
  k->uin = (float)p->u;
  k->rho_in = 1.0f;
  k->ground = p->ground == WT_GROUND_NOSLIP ? 1u : (p->ground == WT_GROUND_MOVING ? 2u : 0u);
  k->sponge_start = (float)(p->sponge_start * nx);
  k->sponge_nu = (float)p->sponge_nu;
  k->u_ground = p->ground == WT_GROUND_MOVING ? (float)p->u : 0.0f;
  k->ema_alpha = (float)p->ema_alpha;
  k->u_ref = (float)(p->u > 1e-4 ? p->u : 1e-4);
  k->ref_x = nx - 1 < 4u ? nx - 1 : 4u;
  k->side_mode = p->sides == WT_SIDES_PERIODIC ? 1u : 0u;
  k->collision = p->collision == WT_COLL_BGK ? 1u : 0u;
  k->tau_wall = (float)p->tau_wall;
  k->sponge_in = (float)(p->sponge_in * nx);
  k->contact_h = 2.0f;
  k->interp = p->interp ? 1u : 0u;
  return WT_OK;
}

int wt_fits(const wt_dims* d, int32_t precision, int64_t* bytes_needed, int32_t* fits) {
  if (!dims_ok(d) || precision < 0 || precision > 2) return fail(nullptr, WT_E_INVALID, "wt_fits: bad dims/precision");
  const int64_t b = bytes_for(d, precision);
  if (bytes_needed) *bytes_needed = b;
  if (fits) {
    size_t fr = 0, tot = 0;
    cudaError_t e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaMemGetInfo");
    *fits = (int64_t)fr > b + (b >> 3) ? 1 : 0;
  }
  return WT_OK;
}

int wt_create(const wt_dims* d, const wt_params* p, wt_solver** out) {
  if (!out) return fail(nullptr, WT_E_INVALID, "wt_create: out is NULL");
  *out = nullptr;
  if (!p || !dims_ok(d)) return fail(nullptr, WT_E_INVALID, "wt_create: bad dims (need nx,ny,nz >= 1, ny,nz <= 65535, cells < 2^32)");
  if (p->precision < 0 || p->precision > 2) return fail(nullptr, WT_E_INVALID, "wt_create: bad precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(nullptr, WT_E_NO_DEVICE, "wt_create: no CUDA device visible");
  }
  wt_solver* s = new (std::nothrow) wt_solver();
  if (!s) return fail(nullptr, WT_E_OOM, "wt_create: host allocation failed");
  cudaGetDevice(&s->device);
  s->dims = *d;
  s->params = *p;
  s->prec = p->precision;
  s->is3d = d->nz > 1;
  s->q = s->is3d ? 19 : 9;
  s->n = (size_t)d->nx * d->ny * d->nz;
  s->pop_elem = elem_bytes(s->prec);
  wt_pack_params(d, p, &s->kp);
  if (!s->launch_explicit) s->sc_kernel = p->collision == WT_COLL_BGK ? 0 : 4;
  std::string where;
  auto alloc = [&](void** ptr, size_t bytes, const char* name) -> bool {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
      where = std::string("cudaMalloc(") + name + ", " + std::to_string(bytes) + " B): " + cudaGetErrorString(e);
      cudaGetLastError();
      return false;
    }
    return true;
  };
  const size_t fbytes = (size_t)s->q * s->n * s->pop_elem;
  if (cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess ||
      s->num_sms <= 0) {
    cudaGetLastError();
    s->num_sms = 148;
  }
  // one macro block per 256 cells up to 4096 blocks (several cells per thread beyond: the block
  // reductions amortise and the final reduce reads at most 320 KB), one MACRO_SLOTS-double partial each
  s->partial_blocks = (int)std::min<size_t>((s->n + 255) / 256, 4096);
  bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess &&
            create_priority_stream(&s->aux) == cudaSuccess &&
            cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) == cudaSuccess &&
            alloc(&s->f[0], fbytes, "populations A") && alloc(&s->f[1], fbytes, "populations B") &&
            alloc((void**)&s->flags, s->n * 4, "flags") && alloc((void**)&s->sdf, s->n * 4, "sdf") &&
            alloc((void**)&s->cls, s->n, "cell class") && alloc((void**)&s->vel, s->n * 8, "velocity") &&
            alloc((void**)&s->meanA, s->n * 16, "meanA") && alloc((void**)&s->meanB, s->n * 4, "meanB") &&
            alloc((void**)&s->partials, (size_t)s->partial_blocks * RESULT_BYTES, "partials") &&
            alloc((void**)&s->result_dev, RESULT_BYTES, "result") && alloc((void**)&s->err_dev, 4, "error word") &&
            alloc((void**)&s->bnd_count, 4, "boundary counter") &&
            alloc((void**)&s->smp_sets, wt::SMP_SETS_BYTES, "sampling accumulators") &&
            alloc((void**)&s->ps_bar, wt::PS_BAR_WORDS * sizeof(unsigned), "barrier words");
  if (ok && (cudaMallocHost((void**)&s->result_host, RESULT_BYTES) != cudaSuccess ||
             cudaMallocHost((void**)&s->err_host, 4) != cudaSuccess ||
             cudaMallocHost((void**)&s->bnd_count_host, 4) != cudaSuccess)) {
    where = "cudaMallocHost(result)";
    ok = false;
  }
  if (!ok) {
    int code = where.find("out of memory") != std::string::npos ? WT_E_OOM : WT_E_CUDA;
    free_all(s);
    delete s;
    return fail(nullptr, code, "wt_create: " + (where.empty() ? std::string("stream creation failed") : where));
  }
  cudaMemsetAsync(s->flags, 0, s->n * 4, s->stream);
  cudaMemsetAsync(s->sdf, 0, s->n * 4, s->stream);
  cudaMemsetAsync(s->vel, 0, s->n * 8, s->stream);
  cudaMemsetAsync(s->err_dev, 0, 4, s->stream);
  *s->err_host = 0;
  k_clear_stats<<<grid_for(s->n), 256, 0, s->stream>>>(s->meanA, s->meanB, s->n);
  s->launches++;
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    std::string m = std::string("wt_create: ") + cudaGetErrorString(e);
    free_all(s);
    delete s;
    return fail(nullptr, WT_E_CUDA, m);
  }
  s->pending_init = true;
  s->cls_dirty = true;
  *out = s;
  return WT_OK;
}

void wt_destroy(wt_solver* s) {
  if (!s) return;
  DeviceGuard g(s->device);
  for (cudaStream_t st : {s->stream, s->aux, s->copy_up, s->copy_rd})
    if (st) cudaStreamSynchronize(st);
  free_all(s);
  delete s;
}

const char* wt_last_error(const wt_solver* s) { return s ? s->err.c_str() : g_create_err.c_str(); }

int wt_set_params(wt_solver* s, const wt_params* p) {
  if (!s || !p) return WT_E_INVALID;
  if (p->precision != s->prec) return fail(s, WT_E_INVALID, "wt_set_params: precision is fixed at creation");
  s->params = *p;
  wt_pack_params(&s->dims, p, &s->kp);
  if (!s->launch_explicit) s->sc_kernel = p->collision == WT_COLL_BGK ? 0 : 4;
  invalidate_graphs(s);
  s->tab_dirty = true;
  return WT_OK;
}

int wt_get_params(const wt_solver* s, wt_params* out) {
  if (!s || !out) return WT_E_INVALID;
  *out = s->params;
  return WT_OK;
}

int wt_get_kparams(const wt_solver* s, wt_kparams* out) {
  if (!s || !out) return WT_E_INVALID;
  *out = s->kp;
  return WT_OK;
}

int wt_reset(wt_solver* s) {
  if (!s) return WT_E_INVALID;
  s->pending_init = true;
  s->step_count = 0;
  return wt_clear_stats(s);
}

int wt_clear_stats(wt_solver* s) {
  if (!s) return WT_E_INVALID;
  DeviceGuard g(s->device);
  k_clear_stats<<<grid_for(s->n), 256, 0, s->stream>>>(s->meanA, s->meanB, s->n);
  s->launches++;
  WT_CUDA(s, cudaGetLastError(), "clear_stats");
  return WT_OK;
}

int64_t wt_step_count(const wt_solver* s) { return s ? s->step_count : -1; }

// The difference words: one per comparison (0: synchronous uploads, 1 and 2: the asynchronous
// flags and wall-distance uploads), on the device and in mapped page-locked host memory.
enum { DIFF_SYNC = 0, DIFF_FLAGS = 1, DIFF_SDF = 2, DIFF_WORDS = 4 };
static int ensure_diff(wt_solver* s) {
  if (s->diff_host_dev) return WT_OK;
  if ((!s->diff_dev && cudaMalloc((void**)&s->diff_dev, DIFF_WORDS * 4) != cudaSuccess) ||
      (!s->diff_host && cudaMallocHost((void**)&s->diff_host, DIFF_WORDS * 4) != cudaSuccess)) {
    cudaGetLastError();
    return fail(s, WT_E_OOM, "upload comparison words");
  }
  WT_CUDA(s, cudaMemset(s->diff_dev, 0, DIFF_WORDS * 4), "upload comparison words");
  WT_CUDA(s, cudaHostGetDevicePointer((void**)&s->diff_host_dev, s->diff_host, 0), "upload comparison words");
  return WT_OK;
}

// queues the comparison of *staged with *cur on `st`: difference word w lands in diff_host[w]
static cudaError_t queue_compare(wt_solver* s, const uint32_t* staged, const uint32_t* cur, int w, cudaStream_t st) {
  k_diff_words<<<grid_for(s->n), 256, 0, st>>>(staged, cur, s->n, s->diff_dev + w);
  k_take_word<<<1, 1, 0, st>>>(s->diff_dev + w, s->diff_host_dev + w);
  s->launches += 2;
  return cudaGetLastError();
}
static bool differs(const wt_solver* s, int w) { return reinterpret_cast<volatile uint32_t*>(s->diff_host)[w] != 0u; }

// Compares the staged upload with *cur on the device; when they differ the stage becomes the
// current buffer (the old one becomes the stage) and `changed` is set.
static int commit_stage(wt_solver* s, uint32_t** cur, bool* changed, const char* what) {
  WT_CUDA(s, queue_compare(s, s->stage, *cur, DIFF_SYNC, s->stream), what);
  WT_CUDA(s, cudaStreamSynchronize(s->stream), what);
  *changed = differs(s, DIFF_SYNC);
  if (*changed) std::swap(*cur, s->stage);
  return WT_OK;
}

static int ensure_stage(wt_solver* s) {
  int rc = ensure_diff(s);
  if (rc || s->stage) return rc;
  if (cudaMalloc((void**)&s->stage, s->n * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(s, WT_E_OOM, "upload staging buffer");
  }
  return WT_OK;
}

// Applies the asynchronous uploads staged since the last call. Each was compared with the current
// buffer on the upload copy stream right after its copy (the comparison runs while the steps
// before it run), so applying one needs no round trip through the compute stream: once the
// copies and comparisons are done, a staged buffer that differs becomes the current one (flags
// first, then wall distances, as the synchronous uploads would have). Every call that reads or
// writes the geometry runs this first, so an asynchronous upload is seen by everything queued
// after it. A buffer that stops being current may still be read by steps in flight: the next
// upload into it waits for them (ev_swap).
static int settle_uploads(wt_solver* s) {
  if (!s->up_flags && !s->up_sdf) return WT_OK;
  WT_CUDA(s, cudaEventSynchronize(s->ev_up), "apply uploads");
  bool swapped = false;
  if (s->up_flags) {
    s->up_flags = false;
    if (differs(s, DIFF_FLAGS)) {
      std::swap(s->flags, s->stage_flags);
      s->cls_dirty = true;
      swapped = true;
    }
  }
  if (s->up_sdf) {
    s->up_sdf = false;
    if (differs(s, DIFF_SDF)) {
      std::swap(s->sdf, s->stage_sdf);
      s->tab_dirty = true;  // the wall distances set the link records, and the graphs hold the buffer
      swapped = true;
    }
  }
  if (swapped) {
    WT_CUDA(s, cudaEventRecord(s->ev_swap, s->stream), "apply uploads");
    s->swap_pending = true;
  }
  return WT_OK;
}

// the copy streams and events of the asynchronous calls, created on first use
static int ensure_async(wt_solver* s) {
  if (s->copy_up) return WT_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&s->copy_rd, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_up, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_src, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_rd, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_smp, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_swap, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_up, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(s, e, "asynchronous copy streams");
  return WT_OK;
}

// Kernels that write the velocity field wait for the asynchronous readbacks issued before them.
static int order_after_reads(wt_solver* s) {
  if (s->rd_issued) WT_CUDA(s, cudaStreamWaitEvent(s->stream, s->ev_rd, 0), "order after readback");
  return WT_OK;
}

static int no_pending_sample(wt_solver* s, const char* what) {
  if (!s->sample_pending) return WT_OK;
  return fail(s, WT_E_STATE, std::string(what) + ": an asynchronous sample is pending (call wt_sample_wait first)");
}

int wt_upload_flags(wt_solver* s, const uint32_t* flags, int64_t n) {
  if (!s || !flags) return WT_E_INVALID;
  if ((size_t)n != s->n) return fail(s, WT_E_INVALID, "wt_upload_flags: n != nx*ny*nz");
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (!rc) rc = ensure_stage(s);
  if (rc) return rc;
  WT_CUDA(s, cudaMemcpyAsync(s->stage, flags, s->n * 4, cudaMemcpyHostToDevice, s->stream), "upload flags");
  bool changed = false;
  rc = commit_stage(s, &s->flags, &changed, "upload flags");
  if (rc) return rc;
  if (changed) s->cls_dirty = true;
  return WT_OK;
}

int wt_upload_sdf(wt_solver* s, const float* d, int64_t n) {
  if (!s || !d) return WT_E_INVALID;
  if ((size_t)n != s->n) return fail(s, WT_E_INVALID, "wt_upload_sdf: n != nx*ny*nz");
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (!rc) rc = ensure_stage(s);
  if (rc) return rc;
  WT_CUDA(s, cudaMemcpyAsync(s->stage, d, s->n * 4, cudaMemcpyHostToDevice, s->stream), "upload sdf");
  k_encode_sdf<<<grid_for(s->n), 256, 0, s->stream>>>(s->stage, s->n);
  s->launches++;
  WT_CUDA(s, cudaGetLastError(), "encode sdf");
  bool changed = false;
  rc = commit_stage(s, &s->sdf, &changed, "upload sdf");
  if (rc) return rc;
  // the wall distances set the Bouzidi fractions of the link records, and the graphs hold the
  // buffer's address
  if (changed) s->tab_dirty = true;
  return WT_OK;
}

// One staged asynchronous upload, queued on copy_up: the copy into the stage, the sdf encoding
// (wall distances) and the comparison with the current buffer; settle_uploads applies it.
static int upload_async(wt_solver* s, bool sdf, const void* src, int64_t n, const char* what) {
  if ((size_t)n != s->n) return fail(s, WT_E_INVALID, std::string(what) + ": n != nx*ny*nz");
  DeviceGuard g(s->device);
  int rc = ensure_async(s);
  if (!rc) rc = ensure_diff(s);
  if (rc) return rc;
  uint32_t** stage = sdf ? &s->stage_sdf : &s->stage_flags;
  if (!*stage) WT_CUDA(s, cudaMalloc((void**)stage, s->n * 4), "cudaMalloc(upload stage)");
  // a stage that was the current buffer until the last swap: steps queued before it may read it
  if (s->swap_pending) {
    WT_CUDA(s, cudaStreamWaitEvent(s->copy_up, s->ev_swap, 0), what);
    s->swap_pending = false;
  }
  WT_CUDA(s, cudaMemcpyAsync(*stage, src, s->n * 4, cudaMemcpyHostToDevice, s->copy_up), what);
  if (sdf) {
    k_encode_sdf<<<grid_for(s->n), 256, 0, s->copy_up>>>(*stage, s->n);
    s->launches++;
  }
  WT_CUDA(s, queue_compare(s, *stage, sdf ? s->sdf : s->flags, sdf ? DIFF_SDF : DIFF_FLAGS, s->copy_up), what);
  WT_CUDA(s, cudaEventRecord(s->ev_up, s->copy_up), what);
  (sdf ? s->up_sdf : s->up_flags) = true;
  return WT_OK;
}

int wt_upload_flags_async(wt_solver* s, const uint32_t* flags, int64_t n) {
  if (!s || !flags) return WT_E_INVALID;
  return upload_async(s, false, flags, n, "wt_upload_flags_async");
}

int wt_upload_sdf_async(wt_solver* s, const float* d, int64_t n) {
  if (!s || !d) return WT_E_INVALID;
  return upload_async(s, true, d, n, "wt_upload_sdf_async");
}

int wt_set_wheels(wt_solver* s, const wt_wheel* w, int32_t count) {
  if (!s || (count > 0 && !w) || count < 0) return WT_E_INVALID;
  invalidate_graphs(s);
  s->tab_dirty = true;
  std::memset(&s->wheels, 0, sizeof s->wheels);
  const int n = count < 16 ? count : 16;
  s->wheels.count = (uint32_t)n;
  for (int k = 0; k < n; k++) {
    const double r = w[k].r > 1e-3 ? w[k].r : 1e-3;
    s->wheels.w[2 * k] = make_float4((float)w[k].c[0], (float)w[k].c[1], (float)w[k].c[2], (float)(1.0 / r));
    s->wheels.w[2 * k + 1] = make_float4((float)w[k].axis[0], (float)w[k].axis[1], (float)w[k].axis[2], (float)w[k].hw);
  }
  return WT_OK;
}

int wt_set_closure(wt_solver* s, const wt_closure* c) {
  if (!s) return WT_E_INVALID;
  DeviceGuard g(s->device);
  if (c == nullptr) {
    if (s->closure_dev) {
      invalidate_graphs(s);
      WT_CUDA(s, cudaStreamSynchronize(s->stream), "wt_set_closure");
      cudaFree(s->closure_dev);
      s->closure_dev = nullptr;
    }
    return WT_OK;
  }
  if (!s->is3d || s->prec == WT_PREC_F64)
    return fail(s, WT_E_UNSUPPORTED, "wt_set_closure: the learned closure needs a D3Q19 handle with f16 or f32 storage");
  if (s->dims.nx % 2 != 0 || s->dims.ny < 2 || s->dims.nz < 2 || (uint64_t)s->q * (uint64_t)s->n >= (1ull << 32))
    return fail(s, WT_E_UNSUPPORTED, "wt_set_closure: the learned closure needs an even nx, ny >= 2, nz >= 2 and "
                                     "19 n < 2^32");
  const float* v = reinterpret_cast<const float*>(c);
  for (size_t k = 0; k < sizeof(wt_closure) / sizeof(float); k++)
    if (!std::isfinite(v[k])) return fail(s, WT_E_INVALID, "wt_set_closure: non-finite network value");
  if (!(c->nu_scale >= 0.0f)) return fail(s, WT_E_INVALID, "wt_set_closure: nu_scale must be >= 0");
  wt::ClosureDev host;
  std::memset(&host, 0, sizeof host);
  wt::closure_pack(*c, host);
  // the captured step graphs carry the network's by-value part: rebuild them
  invalidate_graphs(s);
  if (!s->closure_dev) WT_CUDA(s, cudaMalloc((void**)&s->closure_dev, sizeof(wt::ClosureDev)), "wt_set_closure");
  WT_CUDA(s, cudaMemcpyAsync(s->closure_dev, &host, sizeof host, cudaMemcpyHostToDevice, s->stream), "wt_set_closure");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "wt_set_closure");
  s->closure_host = *c;
  s->closure_p = wt::closure_params(*c);
  return WT_OK;
}

int wt_get_closure(const wt_solver* s, wt_closure* out, int32_t* enabled) {
  if (!s) return WT_E_INVALID;
  if (enabled) *enabled = s->closure_dev != nullptr ? 1 : 0;
  if (out) {
    if (s->closure_dev) *out = s->closure_host;
    else std::memset(out, 0, sizeof *out);
  }
  return WT_OK;
}

int wt_voxelize(wt_solver* s, const float* pos, int64_t nverts, const uint32_t* idx, int64_t ntri, const float m[16],
                const wt_wheel* wheels, int32_t nwheels, wt_voxel_info* info) {
  if (!s || !info || !m || ntri < 0 || nverts < 0 || (ntri > 0 && (!pos || !idx))) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);  // staged uploads land before the voxelizer overwrites the geometry
  if (!rc) rc = wt_set_wheels(s, wheels, nwheels);
  if (rc) return rc;
  std::memset(info, 0, sizeof *info);
  if (ntri == 0) {
    WT_CUDA(s, cudaMemsetAsync(s->flags, 0, s->n * 4, s->stream), "voxelize clear");
    WT_CUDA(s, cudaMemsetAsync(s->sdf, 0, s->n * 4, s->stream), "voxelize clear");
    WT_CUDA(s, cudaStreamSynchronize(s->stream), "voxelize clear");
    s->cls_dirty = true;
    return WT_OK;
  }
  for (int64_t i = 0; i < 3 * ntri; i++)
    if ((int64_t)idx[i] >= nverts) return fail(s, WT_E_INVALID, "wt_voxelize: index out of range of the vertex array");
  // mesh buffers are kept by the handle and grown when a larger mesh arrives
  auto grow = [&](void** buf, size_t* cap, size_t bytes) -> cudaError_t {
    if (bytes <= *cap) return cudaSuccess;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(buf, bytes);
    if (e == cudaSuccess) *cap = bytes;
    return e;
  };
  cudaError_t e = cudaSuccess;
  if ((e = grow(&s->vox_pos, &s->vox_pos_cap, (size_t)nverts * 12 + 16)) != cudaSuccess ||
      (e = grow(&s->vox_idx, &s->vox_idx_cap, (size_t)ntri * 12 + 16)) != cudaSuccess ||
      (!s->vox_info && (e = cudaMalloc((void**)&s->vox_info, 32)) != cudaSuccess))
    return cuda_fail(s, e, "wt_voxelize: mesh buffers");
  // the crossing counters (3 n i32) and vote words (n u32) live in the population buffer that the
  // next step writes in full (16 B per cell; a buffer holds at least 18): the geometry change
  // below makes that step rewrite the solid cells as well, and a pending initialisation rewrites
  // both buffers
  void* dpos = s->vox_pos;
  void* didx = s->vox_idx;
  void* dinfo = s->vox_info;
  void* hits = s->f[s->parity ^ 1];
  void* vote = (char*)hits + 3 * s->n * 4;
  const uint32_t info_init[8] = {0, 0, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0, 0, 0};
  uint32_t info_h[8];
  wt::VoxelJob job;
  job.pos = (const float*)dpos;
  job.idx = (const uint32_t*)didx;
  job.ntri = ntri;
  std::memcpy(job.M, m, sizeof job.M);
  job.hits = (int32_t*)hits;
  job.vote = (uint32_t*)vote;
  job.info = (uint32_t*)dinfo;
  if ((e = cudaMemcpyAsync(dpos, pos, (size_t)nverts * 12, cudaMemcpyHostToDevice, s->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(didx, idx, (size_t)ntri * 12, cudaMemcpyHostToDevice, s->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dinfo, info_init, 32, cudaMemcpyHostToDevice, s->stream)) != cudaSuccess ||
      (e = wt::launch_voxelize(s, job)) != cudaSuccess ||
      (e = cudaMemcpyAsync(info_h, dinfo, 32, cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s->stream)) != cudaSuccess) {
    cudaStreamSynchronize(s->stream);
    s->cls_dirty = true;
    return cuda_fail(s, e, "wt_voxelize");
  }
  s->cls_dirty = true;
  const bool ok = info_h[1] > 0;
  info->frontal = (int32_t)info_h[0];
  info->solid_cells = (int32_t)info_h[1];
  for (int k = 0; k < 3; k++) {
    info->min[k] = ok ? (int32_t)info_h[2 + k] : 0;
    info->max[k] = ok ? (int32_t)info_h[5 + k] + 1 : 0;
  }
  return WT_OK;
}

int wt_step(wt_solver* s, int32_t steps) {
  if (!s || steps < 0) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (!rc) rc = ensure_classified(s);
  if (!rc) rc = ensure_init(s);
  if (rc) return rc;
  int32_t k = 0;
  // single steps until both buffers hold the rest state in their solid cells (the steps that
  // write it are not part of the captured graphs)
  for (; k < steps && !(s->solid_ok[0] && s->solid_ok[1]); k++) {
    cudaError_t e = wt::launch_stream_collide(s, s->f[s->parity], s->f[s->parity ^ 1]);
    if (e != cudaSuccess) return cuda_fail(s, e, "stream_collide");
    s->parity ^= 1;
  }
  if (steps - k >= 2 && s->sc_kernel == WT_LAUNCH_PERSISTENT && wt::persistent_ok(s)) {
    // every remaining step in one cooperative launch of the persistent kernel
    wt_solver* one[1] = {s};
    WT_CUDA(s, wt::launch_persistent(one, 1, steps - k, s->ps_bar, s->err_dev, s->stream), "persistent steps");
    s->launches++;
    if ((steps - k) & 1) s->parity ^= 1;
    k = steps;
  }
  if (steps - k >= 2 * WT_LONG_PAIRS) {
    // runs of WT_LONG_PAIRS step pairs replay one long graph (fewer graph launches)
    if (!s->long_graph[s->parity]) {
      rc = capture_steps(s, s->parity, WT_LONG_PAIRS, &s->long_graph[s->parity], &s->long_graph_launches);
      if (rc) return rc;
    }
    for (; k + 2 * WT_LONG_PAIRS <= steps; k += 2 * WT_LONG_PAIRS) {
      WT_CUDA(s, cudaGraphLaunch(s->long_graph[s->parity], s->stream), "step graph");
      s->launches += s->long_graph_launches;
    }
  }
  if (steps - k >= 2) {
    // pairs of steps replay the captured ping-pong graph of the current parity
    if (!s->step_graph[s->parity]) {
      rc = capture_step_graph(s, s->parity);
      if (rc) return rc;
    }
    for (; k + 2 <= steps; k += 2) {
      WT_CUDA(s, cudaGraphLaunch(s->step_graph[s->parity], s->stream), "step graph");
      s->launches += s->graph_launches;
    }
  }
  for (; k < steps; k++) {
    cudaError_t e = wt::launch_stream_collide(s, s->f[s->parity], s->f[s->parity ^ 1]);
    if (e != cudaSuccess) return cuda_fail(s, e, "stream_collide");
    s->parity ^= 1;
  }
  s->step_count += steps;
  return WT_OK;
}

// Queues the macro pass and the copies of its result and of the error word to pinned memory.
static int enqueue_sample(wt_solver* s) {
  int rc = settle_uploads(s);
  if (!rc) rc = ensure_init(s);
  if (!rc) rc = ensure_classified(s);  // the macro pass reads the class byte
  if (!rc) rc = order_after_reads(s);
  if (rc) return rc;
  WT_CUDA(s, wt::launch_macro(s), "macro");
  WT_CUDA(s, cudaMemcpyAsync(s->result_host, s->result_dev, RESULT_BYTES, cudaMemcpyDeviceToHost, s->stream), "read result");
  WT_CUDA(s, cudaMemcpyAsync(s->err_host, s->err_dev, 4, cudaMemcpyDeviceToHost, s->stream), "read error word");
  s->sample_step = s->step_count;
  return WT_OK;
}

// Queues `steps` steps, the last with the sampling pass fused, and the result copies.
static int enqueue_step_and_sample(wt_solver* s, int32_t steps) {
  if (steps == 0) return enqueue_sample(s);
  int rc = wt_step(s, 0);  // uploads, classification and initialisation
  if (rc) return rc;
  if (!wt::sample_step_ok(s)) {
    rc = wt_step(s, steps);
    return rc ? rc : enqueue_sample(s);
  }
  // The last step runs the sampling pass's per-cell work on what it stores (no second read of the
  // populations), then the wall force and the solid cells, then the final reduction. With solid
  // cells in place in both buffers, the chunk's last WT_SAMPLE_TAIL steps replay one graph.
  // (the persistent launch takes all steps but the last in one launch instead)
  const bool tail = steps >= WT_SAMPLE_TAIL && s->sc_kernel != WT_LAUNCH_PERSISTENT;
  rc = wt_step(s, steps - (tail ? WT_SAMPLE_TAIL : 1));
  if (!rc) rc = order_after_reads(s);  // the sampling step writes the velocity field
  if (rc) return rc;
  if (tail && s->solid_ok[0] && s->solid_ok[1]) {
    if (!s->sample_graph[s->parity]) {
      rc = capture_sample_graph(s, s->parity);
      if (rc) return rc;
    }
    WT_CUDA(s, cudaGraphLaunch(s->sample_graph[s->parity], s->stream), "sample graph");
    s->launches += s->sample_graph_launches;
    s->step_count += WT_SAMPLE_TAIL;
  } else {
    if (tail) {
      rc = wt_step(s, WT_SAMPLE_TAIL - 1);
      if (rc) return rc;
    }
    WT_CUDA(s, wt::launch_sample_step(s, s->f[s->parity], s->f[s->parity ^ 1]), "sampling step");
    s->parity ^= 1;
    s->step_count += 1;
  }
  s->fused_samples++;
  WT_CUDA(s, cudaMemcpyAsync(s->result_host, s->result_dev, RESULT_BYTES, cudaMemcpyDeviceToHost, s->stream),
          "read result");
  WT_CUDA(s, cudaMemcpyAsync(s->err_host, s->err_dev, 4, cudaMemcpyDeviceToHost, s->stream), "read error word");
  s->sample_step = s->step_count;
  return WT_OK;
}

// the result of a completed sample: error word first, then the decoded statistics
static int finish_sample(wt_solver* s, wt_stats* out) {
  if (*s->err_host != 0) return check_err_flag(s);
  decode(s, s->result_host, out);
  return WT_OK;
}

int wt_sample(wt_solver* s, wt_stats* out) {
  if (!s || !out) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = no_pending_sample(s, "wt_sample");
  if (!rc) rc = enqueue_sample(s);
  if (rc) return rc;
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "sample");
  return finish_sample(s, out);
}

int wt_step_and_sample(wt_solver* s, int32_t steps, wt_stats* out) {
  if (!s || !out || steps < 0) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = no_pending_sample(s, "wt_step_and_sample");
  if (!rc) rc = enqueue_step_and_sample(s, steps);
  if (rc) return rc;
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "sample");
  return finish_sample(s, out);
}

int wt_step_and_sample_async(wt_solver* s, int32_t steps) {
  if (!s || steps < 0) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = no_pending_sample(s, "wt_step_and_sample_async");
  if (!rc) rc = ensure_async(s);
  if (!rc) rc = enqueue_step_and_sample(s, steps);
  if (rc) return rc;
  WT_CUDA(s, cudaEventRecord(s->ev_smp, s->stream), "sample event");
  s->sample_pending = true;
  return WT_OK;
}

int wt_sample_wait(wt_solver* s, wt_stats* out) {
  if (!s || !out) return WT_E_INVALID;
  if (!s->sample_pending) return fail(s, WT_E_STATE, "wt_sample_wait: no asynchronous sample is pending");
  DeviceGuard g(s->device);
  s->sample_pending = false;
  WT_CUDA(s, cudaEventSynchronize(s->ev_smp), "sample");
  return finish_sample(s, out);
}

int wt_read_velocity_half4_async(wt_solver* s, void* out_half4, int64_t n) {
  if (!s || !out_half4 || (size_t)n != s->n) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = ensure_async(s);
  if (rc) return rc;
  // the copy starts once everything queued so far on the compute stream has completed
  WT_CUDA(s, cudaEventRecord(s->ev_src, s->stream), "read velocity");
  WT_CUDA(s, cudaStreamWaitEvent(s->copy_rd, s->ev_src, 0), "read velocity");
  WT_CUDA(s, cudaMemcpyAsync(out_half4, s->vel, s->n * 8, cudaMemcpyDeviceToHost, s->copy_rd), "read velocity");
  WT_CUDA(s, cudaEventRecord(s->ev_rd, s->copy_rd), "read velocity");
  s->rd_issued = true;
  return WT_OK;
}

int wt_sync(wt_solver* s) {
  if (!s) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (rc) return rc;
  for (cudaStream_t st : {s->stream, s->aux, s->copy_up, s->copy_rd})
    if (st) WT_CUDA(s, cudaStreamSynchronize(st), "wt_sync");
  return WT_OK;
}

int wt_read_flags(wt_solver* s, uint32_t* out, int64_t n) {
  if (!s || !out || (size_t)n != s->n) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (rc) return rc;
  WT_CUDA(s, cudaMemcpyAsync(out, s->flags, s->n * 4, cudaMemcpyDeviceToHost, s->stream), "read flags");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read flags");
  return WT_OK;
}

int wt_read_sdf(wt_solver* s, uint32_t* out, int64_t n) {
  if (!s || !out || (size_t)n != s->n) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (rc) return rc;
  WT_CUDA(s, cudaMemcpyAsync(out, s->sdf, s->n * 4, cudaMemcpyDeviceToHost, s->stream), "read sdf");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read sdf");
  return WT_OK;
}

int64_t wt_population_bytes(const wt_solver* s) { return s ? (int64_t)(s->q * s->n * s->pop_elem) : -1; }

int wt_read_populations(wt_solver* s, void* out, int64_t bytes) {
  if (!s || !out || bytes != wt_population_bytes(s)) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = ensure_init(s);
  if (rc) return rc;
  WT_CUDA(s, cudaMemcpyAsync(out, s->f[s->parity], (size_t)bytes, cudaMemcpyDeviceToHost, s->stream), "read populations");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read populations");
  return check_err_flag(s);
}

int wt_write_populations(wt_solver* s, const void* in, int64_t bytes) {
  if (!s || !in || bytes != wt_population_bytes(s)) return WT_E_INVALID;
  DeviceGuard g(s->device);
  WT_CUDA(s, cudaMemcpyAsync(s->f[s->parity], in, (size_t)bytes, cudaMemcpyHostToDevice, s->stream), "write populations");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "write populations");
  s->pending_init = false;
  s->solid_ok[s->parity] = false;  // the written solid cells are read as written until rewritten
  return WT_OK;
}

int wt_read_velocity(wt_solver* s, float* out4, int64_t n) {
  if (!s || !out4 || (size_t)n != s->n) return WT_E_INVALID;
  DeviceGuard g(s->device);
  // widened on the device, then one copy into the caller's buffer (fastest when it is pinned)
  if (!s->vel_f32) WT_CUDA(s, cudaMalloc((void**)&s->vel_f32, s->n * 16), "cudaMalloc(velocity readback)");
  k_vel_to_f32<<<grid_for(s->n), 256, 0, s->stream>>>(s->vel, s->vel_f32, s->n);
  s->launches++;
  WT_CUDA(s, cudaGetLastError(), "read velocity");
  WT_CUDA(s, cudaMemcpyAsync(out4, s->vel_f32, s->n * 16, cudaMemcpyDeviceToHost, s->stream), "read velocity");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read velocity");
  return WT_OK;
}

int wt_read_velocity_half4(wt_solver* s, void* out_half4, int64_t n) {
  if (!s || !out_half4 || (size_t)n != s->n) return WT_E_INVALID;
  DeviceGuard g(s->device);
  WT_CUDA(s, cudaMemcpyAsync(out_half4, s->vel, s->n * 8, cudaMemcpyDeviceToHost, s->stream), "read velocity");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read velocity");
  return WT_OK;
}

int wt_read_means(wt_solver* s, float* mean4, float* meanb, int64_t n) {
  if (!s || (size_t)n != s->n) return WT_E_INVALID;
  DeviceGuard g(s->device);
  if (mean4) WT_CUDA(s, cudaMemcpyAsync(mean4, s->meanA, s->n * 16, cudaMemcpyDeviceToHost, s->stream), "read meanA");
  if (meanb) WT_CUDA(s, cudaMemcpyAsync(meanb, s->meanB, s->n * 4, cudaMemcpyDeviceToHost, s->stream), "read meanB");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read means");
  return WT_OK;
}

int wt_derive_fields(wt_solver* s) {
  if (!s) return WT_E_INVALID;
  DeviceGuard g(s->device);
  if (int rc = settle_uploads(s)) return rc;
  for (uint2** b : {&s->dvort, &s->dstat, &s->dmean})
    if (!*b) WT_CUDA(s, cudaMalloc((void**)b, s->n * 8), "cudaMalloc(derived fields)");
  // queued on the handle's stream like the reference's derive dispatch; the reads that follow wait
  WT_CUDA(s, wt::launch_derive(s), "derive fields");
  return WT_OK;
}

int wt_read_derived(wt_solver* s, float* vort4, float* stat4, float* mean4, int64_t n) {
  if (!s || (size_t)n != s->n) return WT_E_INVALID;
  if (!s->dvort) return fail(s, WT_E_STATE, "wt_read_derived: no derived fields yet (call wt_derive_fields)");
  DeviceGuard g(s->device);
  // widened on the device through the export staging buffer, one field at a time
  const size_t need = s->n;
  if (s->exp_cap < need) {
    if (s->exp_buf) cudaFree(s->exp_buf);
    s->exp_buf = nullptr;
    s->exp_cap = 0;
    WT_CUDA(s, cudaMalloc((void**)&s->exp_buf, need * 16), "cudaMalloc(export)");
    s->exp_cap = need;
  }
  const uint2* src[3] = {s->dvort, s->dstat, s->dmean};
  float* dst[3] = {vort4, stat4, mean4};
  for (int k = 0; k < 3; k++) {
    if (!dst[k]) continue;
    WT_CUDA(s, wt::launch_widen_half4(s, src[k], s->exp_buf, s->n), "read derived");
    WT_CUDA(s, cudaMemcpyAsync(dst[k], s->exp_buf, s->n * 16, cudaMemcpyDeviceToHost, s->stream), "read derived");
    WT_CUDA(s, cudaStreamSynchronize(s->stream), "read derived");
  }
  return WT_OK;
}

int wt_export_fields(wt_solver* s, int32_t stride, float* vel4, float* mean4, float* vort4, int64_t points) {
  if (!s || stride < 1) return WT_E_INVALID;
  const int ox = (s->dims.nx + stride - 1) / stride, oy = (s->dims.ny + stride - 1) / stride,
            oz = (s->dims.nz + stride - 1) / stride;
  const int64_t n = (int64_t)ox * oy * oz;
  if (points != n)
    return fail(s, WT_E_INVALID, "wt_export_fields: points != ceil(nx/stride) * ceil(ny/stride) * ceil(nz/stride)");
  int rc = wt_derive_fields(s);
  if (rc) return rc;
  DeviceGuard g(s->device);
  const size_t need = 3 * (size_t)n;
  if (s->exp_cap < need) {
    if (s->exp_buf) cudaFree(s->exp_buf);
    s->exp_buf = nullptr;
    s->exp_cap = 0;
    WT_CUDA(s, cudaMalloc((void**)&s->exp_buf, need * 16), "cudaMalloc(export)");
    s->exp_cap = need;
  }
  WT_CUDA(s, wt::launch_export(s, stride, ox, oy, oz, s->exp_buf), "export fields");
  float* dst[3] = {vel4, mean4, vort4};
  for (int k = 0; k < 3; k++)
    if (dst[k])
      WT_CUDA(s, cudaMemcpyAsync(dst[k], s->exp_buf + k * n, (size_t)n * 16, cudaMemcpyDeviceToHost, s->stream),
              "export fields");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "export fields");
  return WT_OK;
}

static int ensure_export(wt_solver* s, size_t float4s) {
  if (s->exp_cap >= float4s) return WT_OK;
  if (s->exp_buf) cudaFree(s->exp_buf);
  s->exp_buf = nullptr;
  s->exp_cap = 0;
  WT_CUDA(s, cudaMalloc((void**)&s->exp_buf, float4s * 16), "cudaMalloc(export)");
  s->exp_cap = float4s;
  return WT_OK;
}

int wt_streamlines(wt_solver* s, const wt_streamline_params* p, float* pts4, int64_t n) {
  if (!s || !p || !pts4 || n != (int64_t)p->seeds * (int64_t)p->points) return WT_E_INVALID;
  if (p->seeds == 0 || p->points == 0) return WT_OK;
  DeviceGuard g(s->device);
  int rc = settle_uploads(s);
  if (p->use_mean) rc = wt_derive_fields(s);
  if (!rc) rc = ensure_export(s, (size_t)n);
  if (rc) return rc;
  WT_CUDA(s, wt::launch_streamlines(s, *p, s->exp_buf), "streamlines");
  WT_CUDA(s, cudaMemcpyAsync(pts4, s->exp_buf, (size_t)n * 16, cudaMemcpyDeviceToHost, s->stream), "streamlines");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "streamlines");
  return WT_OK;
}

int wt_probes(wt_solver* s, const float* pos4, int32_t count, float* out8) {
  if (!s || count < 0 || count > 8 || (count > 0 && (!pos4 || !out8))) return WT_E_INVALID;
  if (count == 0) return WT_OK;
  int rc = wt_derive_fields(s);
  if (rc) return rc;
  DeviceGuard g(s->device);
  if (!s->probe_buf) WT_CUDA(s, cudaMalloc((void**)&s->probe_buf, 24 * 16), "cudaMalloc(probes)");
  WT_CUDA(s, cudaMemcpyAsync(s->probe_buf, pos4, (size_t)count * 16, cudaMemcpyHostToDevice, s->stream), "probes");
  WT_CUDA(s, wt::launch_probes(s, s->probe_buf, count, s->probe_buf + 8), "probes");
  WT_CUDA(s, cudaMemcpyAsync(out8, s->probe_buf + 8, (size_t)count * 32, cudaMemcpyDeviceToHost, s->stream), "probes");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "probes");
  return WT_OK;
}

static int ensure_tracers(wt_solver* s, uint32_t count, uint32_t trail) {
  if (s->tr_state && s->tr_count == count && s->tr_trail == trail) return WT_OK;
  if (s->tr_state) cudaFree(s->tr_state);
  if (s->tr_hist) cudaFree(s->tr_hist);
  s->tr_state = nullptr;
  s->tr_hist = nullptr;
  s->tr_count = s->tr_trail = 0;
  WT_CUDA(s, cudaMalloc((void**)&s->tr_state, (size_t)(count ? count : 1) * 16), "tracer state");
  WT_CUDA(s, cudaMalloc((void**)&s->tr_hist, (size_t)(count ? count : 1) * (trail ? trail : 1) * 16), "tracer trail");
  WT_CUDA(s, cudaMemsetAsync(s->tr_state, 0, (size_t)(count ? count : 1) * 16, s->stream), "tracer state");
  WT_CUDA(s, cudaMemsetAsync(s->tr_hist, 0, (size_t)(count ? count : 1) * (trail ? trail : 1) * 16, s->stream), "tracer trail");
  s->tr_count = count;
  s->tr_trail = trail;
  return WT_OK;
}

int wt_advect_tracers(wt_solver* s, const wt_tracer_params* p) {
  if (!s || !p) return WT_E_INVALID;
  if (p->trail == 0 || p->head >= p->trail) return fail(s, WT_E_INVALID, "wt_advect_tracers: need trail >= 1 and head < trail");
  if (p->emitter == 1 && p->nozzles == 0) return fail(s, WT_E_INVALID, "wt_advect_tracers: rake emitter needs nozzles >= 1");
  DeviceGuard g(s->device);
  if (int rc = settle_uploads(s)) return rc;
  int rc = ensure_tracers(s, p->count, p->trail);
  if (rc) return rc;
  if (p->count == 0) return WT_OK;
  WT_CUDA(s, wt::launch_tracers(s, *p), "tracers");
  return WT_OK;
}

int wt_read_tracers(wt_solver* s, float* state4, int64_t count, float* hist4, int64_t hist_len) {
  if (!s || count != (int64_t)s->tr_count) return WT_E_INVALID;
  DeviceGuard g(s->device);
  if (state4 && count)
    WT_CUDA(s, cudaMemcpyAsync(state4, s->tr_state, (size_t)count * 16, cudaMemcpyDeviceToHost, s->stream), "read tracers");
  if (hist4) {
    if (hist_len != (int64_t)s->tr_count * s->tr_trail) return fail(s, WT_E_INVALID, "wt_read_tracers: hist_len != count*trail");
    if (hist_len)
      WT_CUDA(s, cudaMemcpyAsync(hist4, s->tr_hist, (size_t)hist_len * 16, cudaMemcpyDeviceToHost, s->stream), "read trail");
  }
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "read tracers");
  return WT_OK;
}

int wt_write_tracers(wt_solver* s, const float* state4, int64_t count, const float* hist4, int64_t hist_len,
                     uint32_t trail) {
  if (!s || count < 0 || trail == 0 || (count > 0 && !state4)) return WT_E_INVALID;
  if (hist4 && hist_len != count * (int64_t)trail) return fail(s, WT_E_INVALID, "wt_write_tracers: hist_len != count*trail");
  DeviceGuard g(s->device);
  int rc = ensure_tracers(s, (uint32_t)count, trail);
  if (rc) return rc;
  if (count) WT_CUDA(s, cudaMemcpyAsync(s->tr_state, state4, (size_t)count * 16, cudaMemcpyHostToDevice, s->stream), "write tracers");
  if (hist4 && hist_len)
    WT_CUDA(s, cudaMemcpyAsync(s->tr_hist, hist4, (size_t)hist_len * 16, cudaMemcpyHostToDevice, s->stream), "write trail");
  WT_CUDA(s, cudaStreamSynchronize(s->stream), "write tracers");
  return WT_OK;
}

int wt_set_launch(wt_solver* s, int32_t kernel, int32_t param, int32_t bx, int32_t by) {
  if (!s) return WT_E_INVALID;
  if (kernel == WT_LAUNCH_ROW_PIPELINE) {
    if (param != 2 || bx != 0 || by < 0 || by > 16)
      return fail(s, WT_E_INVALID, "wt_set_launch: the row pipeline takes param 2, bx 0 and 0..16 rows per block");
  } else if (kernel == WT_LAUNCH_PERSISTENT || kernel == WT_LAUNCH_QUEUE) {
    if (param != 2 || bx != 0 || by != 0)
      return fail(s, WT_E_INVALID, "wt_set_launch: the persistent kernel takes param 2, bx 0, by 0");
    // the work queue's item counter and arrival count start at zero
    DeviceGuard g(s->device);
    WT_CUDA(s, cudaMemsetAsync(s->ps_bar, 0, wt::PS_BAR_WORDS * sizeof(unsigned), s->stream), "wt_set_launch");
  } else if (!(kernel == 0 || (kernel >= 2 && kernel <= 4))) {
    return fail(s, WT_E_INVALID, "wt_set_launch: occupancy hint must be 0 or 2..4 CTAs per SM");
  } else if (!(param == 1 || param == 2 || param == 4) || bx < 0 || by < 0 || bx * by > 256 || (bx % 32) != 0 ||
             ((bx == 0) != (by == 0))) {
    return fail(s, WT_E_INVALID, "wt_set_launch: need v in {1,2,4}, bx % 32 == 0, bx*by <= 256");
  }
  if (kernel == 4 && param == 4)
    return fail(s, WT_E_INVALID, "wt_set_launch: 4 cells per thread supports occupancy hints 0..3");
  s->sc_kernel = kernel;
  s->sc_param = param;
  s->sc_bx = bx;
  s->sc_by = by;
  s->launch_explicit = true;
  invalidate_graphs(s);
  return WT_OK;
}

int wt_set_wait_limit(wt_solver* s, int64_t polls) {
  if (!s) return WT_E_INVALID;
  s->rp_wait_limit = polls < 0 ? (1u << 22) : (uint32_t)std::min<int64_t>(polls, 0xffffffffll);
  invalidate_graphs(s);  // the limit is a kernel argument captured in the step graphs
  return WT_OK;
}

int wt_autotune(wt_solver* s, int32_t iters, int32_t* out4) {
  if (!s || iters < 1) return WT_E_INVALID;
  DeviceGuard g(s->device);
  int rc = ensure_classified(s);
  if (!rc) rc = ensure_init(s);
  if (rc) return rc;
  struct Cand {
    int kernel, param, bx, by;
  };
  std::vector<Cand> cands;
  const bool vec = s->prec == WT_PREC_F16 || s->prec == WT_PREC_F32;
  for (int v : {2, 4}) {
    if (!vec || s->dims.nx % v) continue;
    const int runs = s->dims.nx / v;
    for (int mb : {0, 2, 3, 4}) {
      if (v == 4 && mb == 4) continue;
      for (int bx : {32, 64, 128, 256}) {
        if (bx > ((runs + 31) / 32) * 32) continue;
        for (int threads : {128, 256}) {
          if (threads % bx) continue;
          cands.push_back({mb, v, bx, threads / bx});
        }
      }
    }
  }
  if (wt::rows_pipeline_smem(s) > 0 && s->dims.nx % 2 == 0)
    for (int rows : {2, 4, 8}) cands.push_back({WT_LAUNCH_ROW_PIPELINE, 2, 0, rows});
  cands.push_back({0, 1, 0, 0});
  cudaEvent_t e0, e1;
  WT_CUDA(s, cudaEventCreate(&e0), "autotune");
  WT_CUDA(s, cudaEventCreate(&e1), "autotune");
  float best = 1e30f;
  Cand pick = {s->sc_kernel, s->sc_param, s->sc_bx, s->sc_by};
  for (const Cand& c : cands) {
    s->sc_kernel = c.kernel;
    s->sc_param = c.param;
    s->sc_bx = c.bx;
    s->sc_by = c.by;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; k++) e = wt::launch_stream_collide(s, s->f[s->parity], s->f[s->parity ^ 1]);
    if (e == cudaSuccess) e = cudaEventRecord(e0, s->stream);
    for (int k = 0; k < iters && e == cudaSuccess; k++)
      e = wt::launch_stream_collide(s, s->f[s->parity], s->f[s->parity ^ 1]);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return cuda_fail(s, e, "autotune");
    }
    if (ms < best) {
      best = ms;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s->sc_kernel = pick.kernel;
  s->sc_param = pick.param;
  s->sc_bx = pick.bx;
  s->sc_by = pick.by;
  s->launch_explicit = true;
  invalidate_graphs(s);
  if (out4) {
    out4[0] = pick.kernel;
    out4[1] = pick.param;
    out4[2] = pick.bx;
    out4[3] = pick.by;
  }
  return check_err_flag(s);
}

int wt_get_launch(const wt_solver* s, int32_t* out4) {
  if (!s || !out4) return WT_E_INVALID;
  out4[0] = s->sc_kernel;
  out4[1] = s->sc_param;
  out4[2] = s->sc_bx;
  out4[3] = s->sc_by;
  return WT_OK;
}

void* wt_stream(const wt_solver* s) { return s ? (void*)s->stream : nullptr; }
int32_t wt_device(const wt_solver* s) { return s ? s->device : -1; }
int64_t wt_launch_count(const wt_solver* s) { return s ? s->launches : -1; }
int64_t wt_fused_sample_count(const wt_solver* s) { return s ? s->fused_samples : -1; }

}  // extern "C"

/* ---- batches of tunnels -------------------------------------------------------------------- */
struct wt_batch {
  int device = 0;
  std::vector<wt_solver*> m;
  cudaStream_t stream = nullptr;  // capture origin and replay stream
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_done;
  cudaGraphExec_t graph = nullptr;       // one step pair of every member
  cudaGraphExec_t long_graph = nullptr;  // WT_LONG_PAIRS step pairs
  std::vector<uint64_t> gens;       // member graph generations the graph was captured at
  std::vector<int> parities;        // member parities the graph was captured at
  std::vector<int64_t> per_replay;  // kernel launches of each member inside one replay
  std::vector<int64_t> long_per_replay;
  bool fused = false;  // wt_batch_set_fused(b, 1)
  bool persistent = false;  // wt_batch_set_fused(b, WT_BATCH_PERSISTENT)
  bool queue = false;       // wt_batch_set_fused(b, WT_BATCH_QUEUE)
  unsigned* ps_bar = nullptr;  // the persistent kernel's barrier words
  std::string err;
};

namespace {

int bfail(wt_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  else g_create_err = msg;
  return code;
}

void batch_drop_graph(wt_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->long_graph) cudaGraphExecDestroy(b->long_graph);
  b->graph = nullptr;
  b->long_graph = nullptr;
}

bool batch_graph_current(const wt_batch* b) {
  if (!b->graph) return false;
  for (size_t k = 0; k < b->m.size(); k++)
    if (b->gens[k] != b->m[k]->graph_gen || b->parities[k] != b->m[k]->parity) return false;
  return true;
}

// Whether the batch's steps fuse: every member takes the batch kernel with the same storage and
// collision, and the table holds them all.
bool batch_fused(const wt_batch* b) {
  if (!b->fused || b->m.size() > (size_t)wt::BATCH_MAX_FUSED) return false;
  for (const wt_solver* s : b->m)
    if (!wt::batch_fusable(s) || s->prec != b->m[0]->prec || s->kp.collision != b->m[0]->kp.collision) return false;
  return true;
}

// Whether the members can share the persistent kernel's work queue: same lattice, storage and
// collision for every member, each able to take it, and the table holds them all.
bool batch_queue_ok(const wt_batch* b) {
  if (b->m.size() > 48) return false;
  const wt_solver* s0 = b->m[0];
  for (const wt_solver* s : b->m)
    if (!wt::persistent_ok(s) || s->is3d != s0->is3d || s->prec != s0->prec || s->kp.collision != s0->kp.collision)
      return false;
  return true;
}
// the batch's steps as one cooperative launch per wt_batch_step call (WT_BATCH_PERSISTENT)
bool batch_persistent(const wt_batch* b) { return b->persistent && batch_queue_ok(b); }
// the batch's steps as one launch of the work queue per step, under the batch graphs (WT_BATCH_QUEUE)
bool batch_queue(const wt_batch* b) { return b->queue && batch_queue_ok(b); }

// One step of every member with the bulk rows of all of them in one launch of the batch kernel on
// the batch stream; each member's face rows and wall cells run on its auxiliary stream alongside,
// and join back before the next step.
cudaError_t batch_fused_step(wt_batch* b, int half) {
  wt::BatchTable tab;
  std::memset(&tab, 0, sizeof tab);
  tab.count = (uint32_t)b->m.size();
  uint32_t tiles = 0;
  cudaError_t e = cudaSuccess;
  for (size_t k = 0; k < b->m.size() && e == cudaSuccess; k++) {
    wt_solver* s = b->m[k];
    const int p = s->parity ^ half;
    e = wt::launch_aux_kernels(s, s->f[p], s->f[p ^ 1], b->stream);
    wt::BatchTunnel& t = tab.t[k];
    t.P = s->kp;
    t.fin = s->f[p];
    t.fout = s->f[p ^ 1];
    t.cls = s->cls;
    t.gs = s->gs;
    t.tiles_x = (uint32_t)((s->dims.nx / 2 + wt::BATCH_BX - 1) / wt::BATCH_BX);
    t.tiles_y = (uint32_t)((s->dims.ny + wt::BATCH_BY - 1) / wt::BATCH_BY);
    tab.tile0[k] = tiles;
    tiles += t.tiles_x * t.tiles_y * (uint32_t)s->dims.nz;
  }
  tab.tile0[b->m.size()] = tiles;
  if (e == cudaSuccess) e = wt::launch_batch_bulk(b->m[0]->prec, b->m[0]->kp.collision == 1u, tab, tiles, b->stream);
  if (e == cudaSuccess) b->m[0]->launches++;
  for (size_t k = 0; k < b->m.size() && e == cudaSuccess; k++) e = cudaStreamWaitEvent(b->stream, b->m[k]->ev_join, 0);
  return e;
}

// One graph for two steps of every member. Fused batches: two steps of the batch kernel plus the
// members' face and wall kernels. Otherwise each member's step kernels hang off a fork from the
// batch stream, so independent tunnels run concurrently, and all join back at the end.
int batch_capture_pairs(wt_batch* b, int pairs, cudaGraphExec_t* out, std::vector<int64_t>* per_replay) {
  const size_t n = b->m.size();
  std::vector<int64_t> l0(n);
  for (size_t k = 0; k < n; k++) l0[k] = b->m[k]->launches;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
  if (batch_queue(b)) {
    // one work-queue launch per step; the item counters start from zero in every replay
    e = cudaMemsetAsync(b->ps_bar, 0, wt::PS_BAR_WORDS * sizeof(unsigned), b->stream);
    for (int k = 0; k < 2 * pairs && e == cudaSuccess; k++) {
      e = wt::launch_queue_step(b->m.data(), (int)n, k, b->ps_bar, b->m[0]->err_dev, b->stream);
      if (e == cudaSuccess) b->m[0]->launches++;
    }
  } else if (batch_fused(b)) {
    for (int k = 0; k < pairs && e == cudaSuccess; k++) {
      e = batch_fused_step(b, 0);
      if (e == cudaSuccess) e = batch_fused_step(b, 1);
    }
  } else {
    e = cudaEventRecord(b->ev_fork, b->stream);
    for (size_t k = 0; k < n && e == cudaSuccess; k++) {
      wt_solver* s = b->m[k];
      const int p = s->parity;
      e = cudaStreamWaitEvent(s->stream, b->ev_fork, 0);
      for (int j = 0; j < pairs && e == cudaSuccess; j++) {
        e = wt::launch_stream_collide(s, s->f[p], s->f[p ^ 1]);
        if (e == cudaSuccess) e = wt::launch_stream_collide(s, s->f[p ^ 1], s->f[p]);
      }
      if (e == cudaSuccess) e = cudaEventRecord(b->ev_done[k], s->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->ev_done[k], 0);
    }
  }
  const cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, graph, cudaGraphInstantiateFlagUseNodePriority);
  if (graph) cudaGraphDestroy(graph);
  for (size_t k = 0; k < n; k++) {
    (*per_replay)[k] = b->m[k]->launches - l0[k];
    b->m[k]->launches = l0[k];
  }
  if (e != cudaSuccess) {
    *out = nullptr;
    cudaGetLastError();
    return bfail(b, WT_E_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
  }
  return WT_OK;
}

// the step-pair graph and the long graph, at the members' current generations and parities
int batch_capture(wt_batch* b) {
  batch_drop_graph(b);
  int rc = batch_capture_pairs(b, 1, &b->graph, &b->per_replay);
  if (!rc) rc = batch_capture_pairs(b, WT_LONG_PAIRS, &b->long_graph, &b->long_per_replay);
  if (rc) {
    batch_drop_graph(b);
    return rc;
  }
  for (size_t k = 0; k < b->m.size(); k++) {
    b->gens[k] = b->m[k]->graph_gen;
    b->parities[k] = b->m[k]->parity;
  }
  return WT_OK;
}

int batch_single_step(wt_batch* b) {
  for (wt_solver* s : b->m) {
    cudaError_t e = wt::launch_stream_collide(s, s->f[s->parity], s->f[s->parity ^ 1]);
    if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
    s->parity ^= 1;
  }
  return WT_OK;
}

// orders the batch stream behind all work queued so far on every member's stream
int batch_wait_members(wt_batch* b) {
  for (wt_solver* s : b->m) {
    cudaError_t e = cudaEventRecord(s->ev_join, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, s->ev_join, 0);
    if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
  }
  return WT_OK;
}

}  // namespace

extern "C" {

int wt_batch_create(wt_solver* const* members, int32_t count, wt_batch** out) {
  if (!out) return bfail(nullptr, WT_E_INVALID, "wt_batch_create: out is NULL");
  *out = nullptr;
  if (!members || count < 1) return bfail(nullptr, WT_E_INVALID, "wt_batch_create: need at least one solver");
  for (int32_t k = 0; k < count; k++) {
    if (!members[k]) return bfail(nullptr, WT_E_INVALID, "wt_batch_create: NULL solver");
    if (members[k]->device != members[0]->device)
      return bfail(nullptr, WT_E_INVALID, "wt_batch_create: solvers on different devices");
    for (int32_t j = 0; j < k; j++)
      if (members[j] == members[k]) return bfail(nullptr, WT_E_INVALID, "wt_batch_create: a solver appears twice");
  }
  wt_batch* b = new (std::nothrow) wt_batch();
  if (!b) return bfail(nullptr, WT_E_OOM, "wt_batch_create: host allocation failed");
  b->device = members[0]->device;
  b->m.assign(members, members + count);
  b->gens.assign(count, 0);
  b->parities.assign(count, 0);
  b->per_replay.assign(count, 0);
  b->long_per_replay.assign(count, 0);
  b->ev_done.assign(count, nullptr);
  DeviceGuard g(b->device);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaMalloc((void**)&b->ps_bar, wt::PS_BAR_WORDS * sizeof(unsigned)) == cudaSuccess;
  for (int32_t k = 0; ok && k < count; k++)
    ok = cudaEventCreateWithFlags(&b->ev_done[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    wt_batch_destroy(b);
    return bfail(nullptr, WT_E_CUDA, "wt_batch_create: stream / event creation failed");
  }
  *out = b;
  return WT_OK;
}

void wt_batch_destroy(wt_batch* b) {
  if (!b) return;
  DeviceGuard g(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  if (b->ps_bar) cudaFree(b->ps_bar);
  for (cudaEvent_t e : b->ev_done)
    if (e) cudaEventDestroy(e);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char* wt_batch_last_error(const wt_batch* b) { return b ? b->err.c_str() : g_create_err.c_str(); }

int32_t wt_batch_size(const wt_batch* b) { return b ? (int32_t)b->m.size() : -1; }

int wt_batch_set_fused(wt_batch* b, int32_t on) {
  if (!b) return WT_E_INVALID;
  DeviceGuard g(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  b->fused = on == 1;
  b->persistent = on == WT_BATCH_PERSISTENT;
  b->queue = on == WT_BATCH_QUEUE;
  return WT_OK;
}

int wt_batch_step(wt_batch* b, int32_t steps) {
  if (!b || steps < 0) return WT_E_INVALID;
  DeviceGuard g(b->device);
  for (wt_solver* s : b->m) {
    int rc = settle_uploads(s);
    if (!rc) rc = ensure_classified(s);
    if (!rc) rc = ensure_init(s);
    if (rc) return bfail(b, rc, std::string("member: ") + s->err);
  }
  auto all_solid_ok = [&]() {
    for (wt_solver* s : b->m)
      if (!(s->solid_ok[0] && s->solid_ok[1])) return false;
    return true;
  };
  int32_t k = 0;
  // single steps (all members together) until the solid cells of every buffer hold the rest
  // state: the steps that write it stay out of the graph
  for (; k < steps && !all_solid_ok(); k++) {
    int rc = batch_single_step(b);
    if (rc) return rc;
  }
  if (steps - k >= 2 && batch_persistent(b)) {
    // every remaining step of every member in one cooperative launch of the persistent kernel
    int rc = batch_wait_members(b);
    if (rc) return rc;
    cudaError_t e = wt::launch_persistent(b->m.data(), (int)b->m.size(), steps - k, b->ps_bar, b->m[0]->err_dev,
                                          b->stream);
    if (e == cudaSuccess) e = cudaEventRecord(b->ev_fork, b->stream);
    for (wt_solver* s : b->m)
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s->stream, b->ev_fork, 0);
    if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch persistent steps: ") + cudaGetErrorString(e));
    b->m[0]->launches++;
    if ((steps - k) & 1)
      for (wt_solver* s : b->m) s->parity ^= 1;
    k = steps;
  }
  if (steps - k >= 2) {
    int rc = batch_wait_members(b);
    if (rc) return rc;
    if (!batch_graph_current(b)) {
      rc = batch_capture(b);
      if (rc) return rc;
    }
    for (; k + 2 * WT_LONG_PAIRS <= steps; k += 2 * WT_LONG_PAIRS) {
      cudaError_t e = cudaGraphLaunch(b->long_graph, b->stream);
      if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
      for (size_t j = 0; j < b->m.size(); j++) b->m[j]->launches += b->long_per_replay[j];
    }
    for (; k + 2 <= steps; k += 2) {
      cudaError_t e = cudaGraphLaunch(b->graph, b->stream);
      if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
      for (size_t j = 0; j < b->m.size(); j++) b->m[j]->launches += b->per_replay[j];
    }
    // members' later work waits for the replays
    cudaError_t e = cudaEventRecord(b->ev_fork, b->stream);
    for (wt_solver* s : b->m)
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s->stream, b->ev_fork, 0);
    if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
  }
  for (; k < steps; k++) {
    int rc = batch_single_step(b);
    if (rc) return rc;
  }
  for (wt_solver* s : b->m) s->step_count += steps;
  return WT_OK;
}

int wt_batch_sample(wt_batch* b, wt_stats* out) {
  if (!b || !out) return WT_E_INVALID;
  DeviceGuard g(b->device);
  // the sampling passes of all members are queued first, then read back together
  for (wt_solver* s : b->m) {
    int rc = no_pending_sample(s, "wt_batch_sample");
    if (!rc) rc = settle_uploads(s);
    if (!rc) rc = ensure_init(s);
    if (!rc) rc = ensure_classified(s);
    if (!rc) rc = order_after_reads(s);
    if (rc) return bfail(b, rc, std::string("member: ") + s->err);
    cudaError_t e = wt::launch_macro(s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->result_host, s->result_dev, RESULT_BYTES, cudaMemcpyDeviceToHost, s->stream);
    s->sample_step = s->step_count;
    if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch sample: ") + cudaGetErrorString(e));
  }
  for (size_t k = 0; k < b->m.size(); k++) {
    wt_solver* s = b->m[k];
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return bfail(b, WT_E_CUDA, std::string("batch sample: ") + cudaGetErrorString(e));
    decode(s, s->result_host, &out[k]);
  }
  return WT_OK;
}

}  // extern "C"
