// wt_closure.cuh — the learned LES closure shared by the stream-collide kernels (wt_lbm.cu) and
// the trainer (wt_closure.cu): per-cell features, the network's arithmetic, and the device-side
// copy of a network.
//
// The network (10 -> 32 -> 32 -> 1) and its numerics:
//   x'  = bf16((x - shift) * scale)                     features, padded to 16 with zeros
//   z1  = x' W1 + b1,  h1 = bf16(gelu(z1))              W1 rounded to bf16, f32 accumulation
//   z2  = h1 W2 + b2,  h2 = bf16(gelu(z2))
//   z3  = h2 . w3 + b3,  nu_t = nu_scale * softplus(z3)
//   gelu(x) = x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))   (tanh form; tanh.approx.f32)
// The two 32-wide layers run on tcgen05 tensor cores in the bulk kernel and the trainer; face and
// wall cells evaluate the same network on CUDA cores (closure_nu). Both use the identical gelu,
// bias and rounding steps; they differ only in the order of the f32 accumulations.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include "../../include/wt.h"
#include "wt_umma.cuh"

namespace wt {

constexpr int CL_IN = WT_CLOSURE_IN;    // 10 features
constexpr int CL_K1 = 16;               // layer-1 K, padded for the K = 16 MMA step
constexpr int CL_H = WT_CLOSURE_HID;    // 32 hidden units
constexpr int CL_NPARAM = CL_IN * CL_H + CL_H + CL_H * CL_H + CL_H + CL_H + 1;  // 1441 trainable values

// Device copy of a network. Images are the tcgen05 B operands (N x K, K-major, no swizzle):
// w1img[n = hidden j][k = input], w2img[n = out j][k = in i] (forward), w2timg[n = in i][k = out j]
// (the dH1 = dZ2 W2^T product of the backward pass). The f32 arrays hold the same bf16-rounded
// weights for the CUDA-core path.
struct __align__(128) ClosureDev {
  uint16_t w1img[CL_H * CL_K1];
  uint16_t w2img[CL_H * CL_H];
  uint16_t w2timg[CL_H * CL_H];
  float w1[CL_IN][CL_H];
  float w2[CL_H][CL_H];
  float w3[CL_H];
  float b1[CL_H];
  float b2[CL_H];
  float b3;
  float nu_scale;
  float shift[CL_IN];
  float scale[CL_IN];
};

// bf16 round to nearest even (finite inputs), as a float and as raw bits
__host__ __device__ __forceinline__ uint16_t bf16_bits(float v) {
#if defined(__CUDA_ARCH__)
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
#else
  uint32_t u;
  memcpy(&u, &v, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
#endif
}
__host__ __device__ __forceinline__ float bf16_val(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ __forceinline__ float bf16r(float v) { return bf16_val(bf16_bits(v)); }

__device__ __forceinline__ float tanh_fast(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// gelu, tanh form; explicit roundings so every kernel evaluates it identically
__device__ __forceinline__ float cl_gelu(float x) {
  const float inner = __fmaf_rn(__fmul_rn(0.044715f, __fmul_rn(x, x)), x, x);
  const float t = tanh_fast(__fmul_rn(0.7978845608028654f, inner));
  const float hx = __fmul_rn(0.5f, x);
  return __fmaf_rn(hx, t, hx);
}
// gelu and its derivative
__device__ __forceinline__ float cl_gelu_d(float x, float& d) {
  const float x2 = __fmul_rn(x, x);
  const float inner = __fmaf_rn(__fmul_rn(0.044715f, x2), x, x);
  const float t = tanh_fast(__fmul_rn(0.7978845608028654f, inner));
  const float hx = __fmul_rn(0.5f, x);
  const float du = __fmul_rn(0.7978845608028654f, __fmaf_rn(0.134145f, x2, 1.0f));
  d = __fmaf_rn(__fmul_rn(hx, __fmaf_rn(-t, t, 1.0f)), du, __fmul_rn(0.5f, __fadd_rn(1.0f, t)));
  return __fmaf_rn(hx, t, hx);
}
__device__ __forceinline__ float cl_softplus(float z) { return z > 20.0f ? z : log1pf(expf(z)); }
__device__ __forceinline__ float cl_sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

// wall-distance feature from the sdf word of a cell (~bits(d), 0 = unknown)
__device__ __forceinline__ float cl_wall_dist(uint32_t s) {
  return s == 0u ? WT_CLOSURE_WALL_CAP : fminf(__uint_as_float(~s), WT_CLOSURE_WALL_CAP);
}

// the 10 features of a cell from its moments: non-equilibrium stress Pi (lattice units), density,
// velocity, the handle's molecular tau0 and the wall distance. |S| is the strain rate the
// Smagorinsky relation assigns to |Pi| at Cs = WT_CLOSURE_FEATURE_CS:
//   tau_s = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi| / rho)) / 2,  |S| = 3 |Pi| / (sqrt(2) rho tau_s)
__device__ __forceinline__ void cl_features(float pxx, float pyy, float pzz, float pxy, float pxz, float pyz,
                                            float rho, float ux, float uy, float uz, float tau0, float wall_d,
                                            float (&x)[CL_IN]) {
  float pn = __fmaf_rn(pxx, pxx, __fmaf_rn(pyy, pyy, __fmul_rn(pzz, pzz)));
  pn = __fmaf_rn(2.0f, __fmaf_rn(pxy, pxy, __fmaf_rn(pxz, pxz, __fmul_rn(pyz, pyz))), pn);
  const float piN = __fsqrt_rn(pn);
  const float k = (float)(18.0 * 1.4142135623730951) * (WT_CLOSURE_FEATURE_CS * WT_CLOSURE_FEATURE_CS);
  const float ts = __fmul_rn(0.5f, __fadd_rn(tau0, __fsqrt_rn(__fmaf_rn(tau0, tau0, __fdiv_rn(__fmul_rn(k, piN), rho)))));
  x[0] = pxx;
  x[1] = pyy;
  x[2] = pzz;
  x[3] = pxy;
  x[4] = pxz;
  x[5] = pyz;
  x[6] = __fdiv_rn(__fmul_rn(2.1213203435596424f, piN), __fmul_rn(rho, ts));
  x[7] = wall_d;
  x[8] = rho;
  x[9] = __fsqrt_rn(__fmaf_rn(ux, ux, __fmaf_rn(uy, uy, __fmul_rn(uz, uz))));
}

// normalised, bf16-rounded network input k
__device__ __forceinline__ float cl_input(const ClosureDev& C, const float (&x)[CL_IN], int k) {
  return bf16r(__fmul_rn(__fsub_rn(x[k], C.shift[k]), C.scale[k]));
}

// the whole network on CUDA cores (face and wall cells): nu_t of one cell
static __device__ __noinline__ float closure_nu(const ClosureDev* __restrict__ C, const float* __restrict__ xin) {
  float x[CL_IN];
#pragma unroll
  for (int k = 0; k < CL_IN; k++) x[k] = bf16r(__fmul_rn(__fsub_rn(xin[k], C->shift[k]), C->scale[k]));
  float h1[CL_H];
#pragma unroll 4
  for (int j = 0; j < CL_H; j++) {
    float a = 0.0f;
#pragma unroll
    for (int k = 0; k < CL_IN; k++) a = __fmaf_rn(x[k], C->w1[k][j], a);
    h1[j] = bf16r(cl_gelu(__fadd_rn(a, C->b1[j])));
  }
  float z3 = 0.0f;
#pragma unroll 2
  for (int j = 0; j < CL_H; j++) {
    float a = 0.0f;
#pragma unroll
    for (int i = 0; i < CL_H; i++) a = __fmaf_rn(h1[i], C->w2[i][j], a);
    z3 = __fmaf_rn(bf16r(cl_gelu(__fadd_rn(a, C->b2[j]))), C->w3[j], z3);
  }
  return __fmul_rn(C->nu_scale, cl_softplus(__fadd_rn(z3, C->b3)));
}


// fills the bf16 images and rounded f32 copies of `c` into `d` (host or device)
__host__ __device__ inline void closure_pack(const wt_closure& c, ClosureDev& d) {
  for (int j = 0; j < CL_H; j++)
    for (int k = 0; k < CL_K1; k++) {
      const float v = k < CL_IN ? c.w1[k][j] : 0.0f;
      d.w1img[umma::kmaj_off(j, k, CL_K1) / 2] = bf16_bits(v);
    }
  for (int i = 0; i < CL_H; i++)
    for (int j = 0; j < CL_H; j++) {
      const uint16_t b = bf16_bits(c.w2[i][j]);
      d.w2img[umma::kmaj_off(j, i, CL_H) / 2] = b;
      d.w2timg[umma::kmaj_off(i, j, CL_H) / 2] = b;
      d.w2[i][j] = bf16_val(b);
    }
  for (int k = 0; k < CL_IN; k++)
    for (int j = 0; j < CL_H; j++) d.w1[k][j] = bf16r(c.w1[k][j]);
  for (int j = 0; j < CL_H; j++) {
    d.w3[j] = bf16r(c.w3[j]);
    d.b1[j] = c.b1[j];
    d.b2[j] = c.b2[j];
  }
  d.b3 = c.b3;
  d.nu_scale = c.nu_scale;
  for (int k = 0; k < CL_IN; k++) {
    d.shift[k] = c.shift[k];
    d.scale[k] = c.scale[k];
  }
}

}  // namespace wt
