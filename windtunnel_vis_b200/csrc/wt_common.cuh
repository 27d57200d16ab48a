// wt_common.cuh — lattice tables, population storage policies and small device helpers shared
// by the sm_100a kernels of the wind-tunnel compute path.
//
// Lattice velocity sets follow src/solver/lattice.ts:39-60 of the reference (same direction
// order, so opp / mirror indices and the SoA population layout f[i * N + cell] agree).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/wt.h"

namespace wt {

// ---- compile-time iteration ------------------------------------------------------------------
template <class F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- lattices ------------------------------------------------------------------------------
struct D2Q9 {
  static constexpr int Q = 9;
  static constexpr int DIM = 2;
  static constexpr int c[9][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0},
                                  {1, 1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0}};
  static constexpr double w[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                                  1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
};

struct D3Q19 {
  static constexpr int Q = 19;
  static constexpr int DIM = 3;
  static constexpr int c[19][3] = {{0, 0, 0},   {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                                   {0, 0, 1},   {0, 0, -1},  {1, 1, 0},  {-1, -1, 0}, {1, 0, 1},
                                   {-1, 0, -1}, {0, 1, 1},   {0, -1, -1}, {1, -1, 0}, {-1, 1, 0},
                                   {1, 0, -1},  {-1, 0, 1},  {0, 1, -1}, {0, -1, 1}};
  static constexpr double w[19] = {1.0 / 3,  1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 18,
                                   1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36,
                                   1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
};

// weight of direction I as a scalar constant (usable in device code, unlike the table itself)
template <class L, int I>
struct Wc {
  static constexpr double v = L::w[I];
};

// index of the direction (x, y, z) in lattice L (compile-time)
template <class L>
constexpr int dir_of(int x, int y, int z) {
  for (int k = 0; k < L::Q; k++)
    if (L::c[k][0] == x && L::c[k][1] == y && L::c[k][2] == z) return k;
  return -1;
}
template <class L> constexpr int opp(int i) { return dir_of<L>(-L::c[i][0], -L::c[i][1], -L::c[i][2]); }
template <class L> constexpr int mirY(int i) { return dir_of<L>(L::c[i][0], -L::c[i][1], L::c[i][2]); }
template <class L> constexpr int mirZ(int i) { return dir_of<L>(L::c[i][0], L::c[i][1], -L::c[i][2]); }
template <class L> constexpr int mirYZ(int i) { return dir_of<L>(L::c[i][0], -L::c[i][1], -L::c[i][2]); }

// ---- population storage --------------------------------------------------------------------
// F32: f as float. F16: (f - w_i) as IEEE half (shifted storage), arithmetic in f32.
// F64: f as double, arithmetic in f64 (the plain-method FP64 oracle run on the GPU).
struct StF32 {
  typedef float T;
  typedef float R;
  static constexpr int PREC = WT_PREC_F32;
  __device__ __forceinline__ static R ld(const T* __restrict__ p, size_t o, R /*w*/) { return __ldg(p + o); }
  __device__ __forceinline__ static void st(T* __restrict__ p, size_t o, R v, R /*w*/) { p[o] = v; }
  __device__ __forceinline__ static T solid(R w) { return w; }
  __device__ __forceinline__ static R cvt(T v, R /*w*/) { return v; }
};
// float(h) + w with one rounding (the widening is exact), in one mixed-precision add of sm_100
__device__ __forceinline__ float h2f_add(__half h, float w) {
  float r;
  asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(r) : "h"(__half_as_ushort(h)), "f"(w));
  return r;
}

struct StF16 {
  typedef __half T;
  typedef float R;
  static constexpr int PREC = WT_PREC_F16;
  __device__ __forceinline__ static R ld(const T* __restrict__ p, size_t o, R w) { return h2f_add(__ldg(p + o), w); }
  __device__ __forceinline__ static void st(T* __restrict__ p, size_t o, R v, R w) { p[o] = __float2half_rn(__fsub_rn(v, w)); }
  __device__ __forceinline__ static T solid(R /*w*/) { return __float2half_rn(0.0f); }
  __device__ __forceinline__ static R cvt(T v, R w) { return h2f_add(v, w); }
};
struct StF64 {
  typedef double T;
  typedef double R;
  static constexpr int PREC = WT_PREC_F64;
  __device__ __forceinline__ static R ld(const T* __restrict__ p, size_t o, R /*w*/) { return __ldg(p + o); }
  __device__ __forceinline__ static void st(T* __restrict__ p, size_t o, R v, R /*w*/) { p[o] = v; }
  __device__ __forceinline__ static T solid(R w) { return w; }
  __device__ __forceinline__ static R cvt(T v, R /*w*/) { return v; }
};

// ---- wheels (SolverGPU.setWheels packing, SolverGPU.ts:325-335) ----------------------------
struct Wheels {
  uint32_t count;
  uint32_t pad[3];
  float4 w[32];  // w[2k] = (centre, 1/R), w[2k+1] = (unit axis, half-width)
};

// ---- cell classes (built from the flags by k_classify) --------------------------------------
enum : uint8_t {
  CLS_SOLID = 1,        // flags != 0
  CLS_NEAR_SOLID = 2,   // fluid with at least one in-domain pull source that is solid
  CLS_BELT_STILL = 4,   // floor cell (y = 0) with a non-wheel solid within the tyre contact patch
  CLS_BOUNDARY = CLS_SOLID | CLS_NEAR_SOLID  // bits that send a cell to the per-cell boundary path
};

__host__ __device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}

// seeded noise in [-amp, amp] for velocity component a of `cell` (rest-state initialisation)
__host__ __device__ __forceinline__ float noise_component(uint32_t seed, uint64_t cell, int a, float amp) {
  uint32_t h = pcg_hash((uint32_t)(cell * 3u + (uint64_t)a) ^ pcg_hash(seed ^ (uint32_t)(cell >> 32)));
  float r = (float)(h >> 8) * (1.0f / 16777216.0f);
  return amp * (2.0f * r - 1.0f);
}

}  // namespace wt
