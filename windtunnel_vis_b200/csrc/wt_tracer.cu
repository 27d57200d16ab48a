// wt_tracer.cu — particle tracer advection for sm_100a (the reference's PARTICLES_WGSL,
// src/render/tracers.ts:3-106, with sVel / solidAt from src/render/wgslRender.ts:22-37), and
// the streamline and probe passes (tracers.ts:109-125, 152-200).
//
// One thread per particle: PCG-seeded spawn (inlet band or rake), midpoint RK2 with adaptive
// sub-steps through the FP16 velocity field of the last sample, respawn when a particle leaves
// the tunnel, enters a solid or ages out, and a write of the trail ring buffer.
//
// Velocity sampling restates the reference's linear clamp-to-edge sampler on an rgba16float
// texture (texel centres at k + 0.5) as explicit trilinear interpolation in f32 with full
// precision weights. Compiled with -fmad=false so particle positions are bit-identical to the
// f32 CPU restatement.
#include <cuda_fp16.h>

#include <cstring>

#include "wt_internal.h"

namespace wt {
namespace {

struct TrCtx {
  wt_tracer_params P;
  float dims[4];
  int n[3];
  const uint2* __restrict__ vel;
  const uint32_t* __restrict__ flags;
};

struct Rng {
  uint32_t s;
  __device__ __forceinline__ float next() {
    s = pcg_hash(s);
    return __uint2float_rn(s) / 4294967295.0f;
  }
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float k) { return f3(a.x * k, a.y * k, a.z * k); }

__device__ __forceinline__ bool solid_at(const TrCtx& T, float3 p) {
  int cx = (int)floorf(p.x), cy = (int)floorf(p.y), cz = (int)floorf(p.z);
  if (T.dims[3] > 0.5f) cz = 0;
  if (cx < 0 || cy < 0 || cz < 0 || cx >= T.n[0] || cy >= T.n[1] || cz >= T.n[2]) return false;
  return T.flags[(size_t)cx + (size_t)T.n[0] * ((size_t)cy + (size_t)T.n[1] * cz)] != 0u;
}

__device__ __forceinline__ float4 vel_at(const TrCtx& T, int x, int y, int z) {
  const uint2 pk = __ldg(T.vel + (size_t)x + (size_t)T.n[0] * ((size_t)y + (size_t)T.n[1] * z));
  const __half2 a = *reinterpret_cast<const __half2*>(&pk.x);
  const __half2 b = *reinterpret_cast<const __half2*>(&pk.y);
  const float2 fa = __half22float2(a), fb = __half22float2(b);
  return make_float4(fa.x, fa.y, fb.x, fb.y);
}

__device__ float3 sample_vel(const TrCtx& T, float3 p) {
  float t[3] = {p.x / T.dims[0], p.y / T.dims[1], p.z / T.dims[2]};
  if (T.dims[3] > 0.5f) t[2] = 0.5f;
  int i0[3], i1[3];
  float fr[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float u = t[a] * (float)T.n[a] - 0.5f;
    const float fl = floorf(u);
    fr[a] = u - fl;
    const int k = (int)fl;
    i0[a] = min(max(k, 0), T.n[a] - 1);
    i1[a] = min(max(k + 1, 0), T.n[a] - 1);
  }
  const float4 v000 = vel_at(T, i0[0], i0[1], i0[2]), v100 = vel_at(T, i1[0], i0[1], i0[2]);
  const float4 v010 = vel_at(T, i0[0], i1[1], i0[2]), v110 = vel_at(T, i1[0], i1[1], i0[2]);
  const float4 v001 = vel_at(T, i0[0], i0[1], i1[2]), v101 = vel_at(T, i1[0], i0[1], i1[2]);
  const float4 v011 = vel_at(T, i0[0], i1[1], i1[2]), v111 = vel_at(T, i1[0], i1[1], i1[2]);
  const float gx = 1.0f - fr[0], gy = 1.0f - fr[1], gz = 1.0f - fr[2];
  auto tri = [&](float a000, float a100, float a010, float a110, float a001, float a101, float a011, float a111) {
    const float c00 = a000 * gx + a100 * fr[0];
    const float c10 = a010 * gx + a110 * fr[0];
    const float c01 = a001 * gx + a101 * fr[0];
    const float c11 = a011 * gx + a111 * fr[0];
    const float c0 = c00 * gy + c10 * fr[1];
    const float c1 = c01 * gy + c11 * fr[1];
    return c0 * gz + c1 * fr[2];
  };
  return f3(tri(v000.x, v100.x, v010.x, v110.x, v001.x, v101.x, v011.x, v111.x),
            tri(v000.y, v100.y, v010.y, v110.y, v001.y, v101.y, v011.y, v111.y),
            tri(v000.z, v100.z, v010.z, v110.z, v001.z, v101.z, v011.z, v111.z));
}

__device__ __forceinline__ float3 vel3(const TrCtx& T, float3 p) {
  float3 v = sample_vel(T, p);
  if (T.dims[3] > 0.5f) v.z = 0.0f;
  return v;
}

__device__ float3 spawn(const TrCtx& T, Rng& R) {
  const bool is2D = T.dims[3] > 0.5f;
  if (T.P.emitter == 0u) {
    const float x = 1.0f + R.next() * 2.0f;
    const float y = 0.5f + R.next() * (T.dims[1] - 1.0f);
    const float z3 = 0.5f + R.next() * (T.dims[2] - 1.0f);  // select() evaluates both operands
    return f3(x, y, is2D ? 0.5f : z3);
  }
  const uint32_t lines = T.P.lines > 1u ? T.P.lines : 1u;
  const uint32_t tot = T.P.nozzles * lines;
  uint32_t k = __float2uint_rz(R.next() * (float)tot);
  k = k < tot - 1u ? k : tot - 1u;
  const float t = ((float)(k % T.P.nozzles) + 0.5f) / (float)T.P.nozzles;
  const float l = (float)(k / T.P.nozzles) - 0.5f * (float)(lines - 1u);
  const float3 A = f3(T.P.rake_a[0], T.P.rake_a[1], T.P.rake_a[2]);
  const float3 B = f3(T.P.rake_b[0], T.P.rake_b[1], T.P.rake_b[2]);
  const float3 D = f3(T.P.rake_d[0], T.P.rake_d[1], T.P.rake_d[2]);
  float3 p = add3(add3(mul3(A, 1.0f - t), mul3(B, t)), mul3(D, l));
  const float jx = R.next() - 0.5f;
  const float jy = R.next() - 0.5f;
  const float jz = R.next() - 0.5f;
  p = add3(p, mul3(f3(jx, jy, jz), 0.35f));
  if (is2D) p.z = 0.5f;
  return p;
}

__device__ float3 fill_pos(const TrCtx& T, Rng& R) {
  const bool is2D = T.dims[3] > 0.5f;
  for (int k = 0; k < 8; k++) {
    const float x = 1.0f + R.next() * (T.dims[0] - 2.0f);
    const float y = 0.5f + R.next() * (T.dims[1] - 1.0f);
    const float z3 = 0.5f + R.next() * (T.dims[2] - 1.0f);
    const float3 p = f3(x, y, is2D ? 0.5f : z3);
    if (!solid_at(T, p)) return p;
  }
  return spawn(T, R);
}

__device__ __forceinline__ bool outside(const TrCtx& T, float3 p) {
  if (T.dims[3] > 0.5f) return p.x < 0.0f || p.y < 0.0f || p.x >= T.dims[0] - 1.0f || p.y >= T.dims[1];
  return p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || p.x >= T.dims[0] - 1.0f || p.y >= T.dims[1] || p.z >= T.dims[2];
}

__global__ void __launch_bounds__(128) k_particles(const TrCtx T, float4* __restrict__ state, float4* __restrict__ hist) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const wt_tracer_params& P = T.P;
  if (i >= P.count) return;
  Rng R{pcg_hash(i ^ pcg_hash(P.seed))};
  float4 s = state[i];
  if (P.fill != 0u) {
    if (P.emitter == 0u) {
      const float3 q = fill_pos(T, R);
      s = make_float4(q.x, q.y, q.z, (float)P.trail);
    } else {
      const float3 q = spawn(T, R);
      s = make_float4(q.x, q.y, q.z, -floorf(R.next() * P.max_age));
    }
    state[i] = s;
    for (uint32_t k = 0; k < P.trail; k++) hist[(size_t)k * P.count + i] = make_float4(s.x, s.y, s.z, 0.0f);
    return;
  }
  if (P.advance == 0u) return;
  if (s.w < 0.0f) {
    s.w += 1.0f;
    if (s.w >= 0.0f) {
      const float3 q = spawn(T, R);
      s = make_float4(q.x, q.y, q.z, 0.0f);
    }
  } else {
    float3 p = f3(s.x, s.y, s.z);
    const float3 v0 = vel3(T, p);
    const float disp = sqrtf(v0.x * v0.x + v0.y * v0.y + v0.z * v0.z) * P.steps;
    const uint32_t nsub = (uint32_t)fminf(fmaxf(ceilf(disp / 0.6f), 1.0f), 24.0f);
    const float h = P.steps / (float)nsub;
    for (uint32_t k = 0; k < nsub; k++) {
      const float3 a = vel3(T, p);
      const float3 b = vel3(T, add3(p, mul3(a, 0.5f * h)));
      p = add3(p, mul3(b, h));
    }
    s = make_float4(p.x, p.y, p.z, s.w + 1.0f);
    if (outside(T, p) || solid_at(T, p) || s.w > P.max_age * 4.0f) {
      const float3 q = spawn(T, R);
      s = make_float4(q.x, q.y, q.z, 0.0f);
    }
  }
  state[i] = s;
  hist[(size_t)P.head * P.count + i] = make_float4(s.x, s.y, s.z, 0.0f);
}

// Four channels of a half4 field at p (the same linear clamp-to-edge sampling as sample_vel).
__device__ float4 sample4(const TrCtx& T, const uint2* __restrict__ field, float3 p) {
  float t[3] = {p.x / T.dims[0], p.y / T.dims[1], p.z / T.dims[2]};
  if (T.dims[3] > 0.5f) t[2] = 0.5f;
  int i0[3], i1[3];
  float fr[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float u = t[a] * (float)T.n[a] - 0.5f;
    const float fl = floorf(u);
    fr[a] = u - fl;
    const int k = (int)fl;
    i0[a] = min(max(k, 0), T.n[a] - 1);
    i1[a] = min(max(k + 1, 0), T.n[a] - 1);
  }
  auto at = [&](int x, int y, int z) {
    const uint2 pk = __ldg(field + (size_t)x + (size_t)T.n[0] * ((size_t)y + (size_t)T.n[1] * z));
    const float2 fa = __half22float2(*reinterpret_cast<const __half2*>(&pk.x));
    const float2 fb = __half22float2(*reinterpret_cast<const __half2*>(&pk.y));
    return make_float4(fa.x, fa.y, fb.x, fb.y);
  };
  const float4 v000 = at(i0[0], i0[1], i0[2]), v100 = at(i1[0], i0[1], i0[2]);
  const float4 v010 = at(i0[0], i1[1], i0[2]), v110 = at(i1[0], i1[1], i0[2]);
  const float4 v001 = at(i0[0], i0[1], i1[2]), v101 = at(i1[0], i0[1], i1[2]);
  const float4 v011 = at(i0[0], i1[1], i1[2]), v111 = at(i1[0], i1[1], i1[2]);
  const float gx = 1.0f - fr[0], gy = 1.0f - fr[1], gz = 1.0f - fr[2];
  auto tri = [&](float a000, float a100, float a010, float a110, float a001, float a101, float a011, float a111) {
    const float c00 = a000 * gx + a100 * fr[0];
    const float c10 = a010 * gx + a110 * fr[0];
    const float c01 = a001 * gx + a101 * fr[0];
    const float c11 = a011 * gx + a111 * fr[0];
    const float c0 = c00 * gy + c10 * fr[1];
    const float c1 = c01 * gy + c11 * fr[1];
    return c0 * gz + c1 * fr[2];
  };
  return make_float4(tri(v000.x, v100.x, v010.x, v110.x, v001.x, v101.x, v011.x, v111.x),
                     tri(v000.y, v100.y, v010.y, v110.y, v001.y, v101.y, v011.y, v111.y),
                     tri(v000.z, v100.z, v010.z, v110.z, v001.z, v101.z, v011.z, v111.z),
                     tri(v000.w, v100.w, v010.w, v110.w, v001.w, v101.w, v011.w, v111.w));
}

__device__ __forceinline__ float len3(float3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }

// Streamlines (STREAMLINES_WGSL, src/render/tracers.ts:152-200): one thread per seed; seeds sit
// line by line on parallel rake lines; each step samples the instantaneous (or mean) velocity,
// takes a midpoint step of length h along its direction, and the line ends (w = -1 from then on)
// where it leaves the tunnel, enters a solid or the speed falls below 1e-3 U.
__global__ void __launch_bounds__(64) k_streamlines(const TrCtx T, const wt_streamline_params S,
                                                    const uint2* __restrict__ mean, float U_lat,
                                                    float4* __restrict__ pts) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.seeds) return;
  const bool is2D = T.dims[3] > 0.5f;
  auto vel = [&](float3 p) {
    const float4 v4 = S.use_mean != 0u ? sample4(T, mean, p) : sample4(T, T.vel, p);
    float3 v = f3(v4.x, v4.y, v4.z);
    if (is2D) v.z = 0.0f;
    return v;
  };
  auto outside = [&](float3 p) {
    if (is2D) return p.x < 0.0f || p.y < 0.0f || p.x >= T.dims[0] || p.y >= T.dims[1];
    return p.x < 0.0f || p.y < 0.0f || p.z < 0.0f || p.x >= T.dims[0] || p.y >= T.dims[1] || p.z >= T.dims[2];
  };
  const uint32_t per = S.per_line > 1u ? S.per_line : 1u;
  const float l = (float)(s / per) - 0.5f * (float)(S.seeds / per - 1u);
  const float t = ((float)(s % per) + 0.5f) / (float)per;
  const float3 A = f3(S.rake_a[0], S.rake_a[1], S.rake_a[2]), B = f3(S.rake_b[0], S.rake_b[1], S.rake_b[2]);
  const float3 D = f3(S.rake_d[0], S.rake_d[1], S.rake_d[2]);
  float3 p = add3(add3(mul3(A, 1.0f - t), mul3(B, t)), mul3(D, l));
  if (is2D) p.z = 0.5f;
  bool alive = true;
  const float U = fmaxf(U_lat, 1e-5f);
  for (uint32_t k = 0; k < S.points; k++) {
    const float3 v = vel(p);
    const float sp = len3(v);
    if (alive && (outside(p) || solid_at(T, p) || sp < U * 1e-3f)) alive = false;
    pts[(size_t)s * S.points + k] = make_float4(p.x, p.y, p.z, alive ? sp : -1.0f);
    if (!alive) continue;
    const float3 a = f3(v.x / sp, v.y / sp, v.z / sp);
    const float3 vm = vel(add3(p, mul3(a, 0.5f * S.h)));
    const float lm = len3(vm);
    if (lm < 1e-9f) {
      alive = false;
      continue;
    }
    p = add3(p, mul3(f3(vm.x / lm, vm.y / lm, vm.z / lm), S.h));
  }
}

// Probes (PROBES_WGSL, src/render/tracers.ts:109-125): instantaneous and mean (ux, uy, uz, rho)
// at up to 8 points.
__global__ void __launch_bounds__(32) k_probes(const TrCtx T, const float4* __restrict__ pos, int count,
                                               const uint2* __restrict__ mean, float4* __restrict__ out) {
  const int i = threadIdx.x;
  if (i >= count) return;
  const float4 q = pos[i];
  const float3 p = f3(q.x, q.y, q.z);
  float4 v = sample4(T, T.vel, p);
  float4 m = sample4(T, mean, p);
  if (T.dims[3] > 0.5f) {
    v.z = 0.0f;
    m.z = 0.0f;
  }
  out[2 * i] = v;
  out[2 * i + 1] = m;
}

TrCtx make_ctx(const wt_solver* s) {
  TrCtx T;
  T.dims[0] = (float)s->dims.nx;
  T.dims[1] = (float)s->dims.ny;
  T.dims[2] = (float)s->dims.nz;
  T.dims[3] = s->dims.nz == 1 ? 1.0f : 0.0f;
  T.n[0] = s->dims.nx;
  T.n[1] = s->dims.ny;
  T.n[2] = s->dims.nz;
  T.vel = s->vel;
  T.flags = s->flags;
  return T;
}

}  // namespace

cudaError_t launch_streamlines(wt_solver* s, const wt_streamline_params& p, float4* pts) {
  TrCtx T = make_ctx(s);
  std::memset(&T.P, 0, sizeof T.P);
  k_streamlines<<<(p.seeds + 63) / 64, 64, 0, s->stream>>>(T, p, s->dmean, s->kp.uin, pts);
  s->launches++;
  return cudaGetLastError();
}

cudaError_t launch_probes(wt_solver* s, const float4* pos, int count, float4* out) {
  TrCtx T = make_ctx(s);
  std::memset(&T.P, 0, sizeof T.P);
  k_probes<<<1, 32, 0, s->stream>>>(T, pos, count, s->dmean, out);
  s->launches++;
  return cudaGetLastError();
}

cudaError_t launch_tracers(wt_solver* s, const wt_tracer_params& p) {
  TrCtx T;
  T.P = p;
  T.dims[0] = (float)s->dims.nx;
  T.dims[1] = (float)s->dims.ny;
  T.dims[2] = (float)s->dims.nz;
  T.dims[3] = s->dims.nz == 1 ? 1.0f : 0.0f;
  T.n[0] = s->dims.nx;
  T.n[1] = s->dims.ny;
  T.n[2] = s->dims.nz;
  T.vel = s->vel;
  T.flags = s->flags;
  const unsigned blocks = (p.count + 127) / 128;
  k_particles<<<blocks, 128, 0, s->stream>>>(T, s->tr_state, s->tr_hist);
  s->launches++;
  return cudaGetLastError();
}

}  // namespace wt
